"""Benchmark of the B200 CaMa-Flood physics time step (CMF_PHYSICS_ADVANCE) on the config-1 workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--members M]

One step is one coupling step (one hour of the config-1 forcing): the stage scheme, the CFL
reduction and NT local-inertial sub-steps over the 1440x720-grid network of ~300k cells with
12k bifurcation channels x 5 levels, levees on 10% of cells and 2000 dams.  The case is generated
from a fixed seed in the reference's file formats (synthetic data; no dataset is read).

Metric: cell-substeps/s = sum over steps and members of NSEQALL * NT / time.
  value     device-resident: runoff already in HBM, one CUDA graph per step, CUDA events on the
            library's stream, L2 flushed (256 MiB write) before every timed step;
  e2e       the public API with host buffers: put_runoff (pinned host -> device), advance, and a
            device -> host read of the step's averaged discharge, timed on the host clock.
--impl reference times the reference algorithm's CPU implementation (the oracle restatement with
OpenMP on all host cores; the Fortran reference itself cannot be compiled on this machine).
Under torchrun every rank runs its own member(s) of the ensemble (weak scaling, no collective on
the data path); rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(ROOT, "cama-flood_v4_b200"), os.path.join(ROOT, "oracle")]

METRIC = "cell-steps/s on 1 B200: plain GPU vs surrogate-assisted at <=1% NSE loss; HBM GB/s"
UNIT = "cell-substeps/s"
CASE_CACHE = os.environ.get("CMF_BENCH_CASES", "/tmp/cmf_bench_cases")
SPINUP_STEPS = 24
WORKLOAD = ("config1: 1440x720 grid, 299157 cells, 12k bifurcation x5, levees 10%, 2000 dams, "
            "hourly AR(1) forcing")


# ----------------------------------------------------------------------------------------- setup
def case_dir(name: str = "cfg1") -> str:
    from cmf_b200 import synth

    d = os.path.join(CASE_CACHE, name)
    if not os.path.exists(os.path.join(d, "input_cmf.nam")):
        spec = {"cfg1": lambda: synth.spec_config1(seed=1), "cfg4": lambda: synth.spec_config4(seed=4)}.get(
            name, lambda: synth.spec_config0(seed=0))()
        tmp = d + f".tmp{os.getpid()}"
        synth.write_case(synth.make_case(spec), tmp)
        try:
            os.rename(tmp, d)
        except OSError:
            pass   # another rank won the race; the contents are identical (same seed)
    return d


def runoff_fields(grarea: np.ndarray, nsteps: int, seed: int) -> np.ndarray:
    """Hourly AR(1) phi=0.9 Gaussian-copula Gamma(0.8, 2.5 mm/day) runoff -> m3/s (CONV_RESOL)."""
    from cmf_b200 import synth

    gen = synth.AR1GammaRunoff(grarea.size, seed)
    out = np.empty((nsteps, grarea.size))
    for k in range(nsteps):
        out[k] = np.maximum((gen.next().astype(np.float64) * grarea) / 86400000.0, 0.0)
    return out


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi sampling (every `interval_ms`) around the timed region; every sample carries the
    host time it arrived at, so the summary can be restricted to a window (`mark_start`/`mark_end`)."""

    def __init__(self, device: int, interval_ms: int = 20):
        self.device = device
        self.interval_ms = interval_ms
        self.proc = None
        self.lines = []
        self.window = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", str(self.interval_ms)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line.strip()))

    def wait_first(self, timeout: float = 3.0) -> None:
        """Returns once the first sample arrived (nvidia-smi takes a moment to start)."""
        t0 = time.perf_counter()
        while self.proc and not self.lines and time.perf_counter() - t0 < timeout:
            time.sleep(0.01)

    def mark_load(self):
        """Start of the loaded span (the replay of the timed steps that precedes the timed region)."""
        self.load = time.perf_counter()

    def mark_start(self):
        self.window = [time.perf_counter(), None]

    def mark_end(self):
        if self.window:
            self.window[1] = time.perf_counter()

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self, loaded: bool = False) -> dict:
        """Median SM clock, maximum and throttle reasons over the timed window, or (loaded=True) over
        the whole loaded span from mark_load() to the window's end."""
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = self.lines
        if self.window and self.window[1]:
            # samples that arrived during the marked span (plus one interval of reporting lag)
            lag = self.interval_ms / 1e3
            t0 = getattr(self, "load", None) if loaded else None
            t0 = self.window[0] if t0 is None else t0
            sel = [x for x in lines if t0 <= x[0] <= self.window[1] + lag]
            lines = sel if sel else lines
        for _, ln in lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 8:
                continue
            try:
                sm.append(float(p[1]))
                mx.append(float(p[2]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if p[4 + k].lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def cpu_model() -> str:
    """The host CPU's model string as lscpu prints it."""
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        for ln in out.splitlines():
            if ln.lower().startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except (OSError, subprocess.SubprocessError):
        pass
    return "unknown"


def bench_config(members: int, warmup: int, steps: int) -> dict:
    """The workload description both arms print (identical dicts): the same network, forcing seed
    and timed window of coupling steps."""
    first = SPINUP_STEPS + warmup
    return {"workload": WORKLOAD, "members_per_gpu": members,
            "timed_window": f"coupling steps {first + 1}-{first + steps} of the seeded hourly forcing (seed 1), "
                            f"after {SPINUP_STEPS} spin-up and {warmup} warm-up steps"}


def closure(budgets: list) -> dict:
    """Global mass-balance closure of CALC_WATBAL (src/cmf_ctrl_physics_mod.F90:216-248) over the
    given steps: DERROR = -(STOPRE - STONXT + RIVINF - RIVOUT), DERROR2 = -(STOPRE2 - STONEW2) [m3]."""
    e1 = [abs(-(b["stopre"] - b["stonxt"] + b["rivinf"] - b["rivout"])) for b in budgets]
    e2 = [abs(-(b["stopre2"] - b["stonew2"])) for b in budgets]
    sto = [abs(b["stonew2"]) for b in budgets]
    return {"max_abs_derror_m3": max(e1), "max_abs_derror2_m3": max(e2),
            "max_rel_derror": max(a / max(s, 1e-300) for a, s in zip(e1, sto)),
            "storage_m3": sto[-1], "steps": len(budgets)}


# ----------------------------------------------------------------------------- algorithmic bytes
def phase_bytes(N: int, E: int, L_bar: float, P: int, Lp: int, nlev: int, ndam: int, ldiag: bool) -> dict:
    """Compulsory HBM bytes per launch of each sub-step kernel (every array element the kernel must
    read or write once every sub-step; gathers of neighbour values are L2 reuse and not counted
    again; outputs written on the last sub-step only -- D2RIVVEL, D2RIVINF, D2FLDINF, D2PTHOUT,
    D2OUTFLW, D2FLDARE, D2SFCELV and the runoff average -- are not counted).
      k_flux : static 7x8 (RIVELV ELEVTN NXTDST RIVWTH RIVHGT RIVLEN RIVMAN) + I1NEXT 4 + state reads
               8x8 (RIVDPH RIVDPH_PRE RIVOUT_PRE FLDOUT_PRE FLDSTO FLDDPH FLDSTO_PRE STORGE)
               + writes 2x8 (RIVOUT FLDOUT) = 140 B/cell, + diagnostics: velocity average r/w 16 and
               the previous sub-step's 7 accumulators r/w 112 (rivout fldout outflw daminf averages,
               outflw rivdph storge maxima)                                 = 140 (+128) B/cell
               + per path: endpoints 8, DST 8, skip 4, ELV/WTH/FLW_PRE/FLW 32 x Lp, FLWSUM 8
      k_rate : RIVOUT FLDOUT 16 + CSR 4 + 4/edge + RIVSTO FLDSTO 16 + RATE 8        = 48 B/cell
               + path CSR 8 and FLWSUM 8 per path end
      k_store: RIVOUT FLDOUT RATE 24 + CSR 8 + I1NEXT 4 + RIVSTO FLDSTO RIVDPH FLDFRC RUNOFF 40
               + RIVSTOMAX RIVLEN RIVWTH GRAREA 32 + layers 16 L_bar + writes 10x8 80 (_PRE x4,
               RIVSTO FLDSTO RIVDPH FLDDPH FLDFRC STORGE)                   = 188+16 L_bar
               (the last sub-step's own accumulators, once per outer step, are not counted)
               + levee: index 4/cell + 7 params + LEVSTO r/w + LEVDPH w per levee cell
               + dams: 112 B per dam, paths: FLW r/w 16 x Lp + FLWSUM 16 per path
    k_store walks the upstream lists through a 4-slot table (16 B per cell, one dependent load
    fewer); the count keeps the CSR's compulsory bytes, so the fraction it gives is conservative."""
    flux = N * (140 + (128 if ldiag else 0)) + P * (8 + 8 + 4 + 32 * Lp + 8) + ndam * 112
    rate = N * 48 + (E - N) * 4 + P * 2 * (8 + 8)
    store = N * (188 + 16 * L_bar) + N * 4 + nlev * (7 * 8 + 16 + 8) + ndam * 112 + P * (16 * Lp + 16)
    return {"k_flux": flux, "k_rate": rate, "k_store": store}


def mean_layers(state: dict, fldstomax: np.ndarray, rivstomax: np.ndarray, N: int, L: int) -> float:
    """Mean floodplain layers the stage scheme scans per cell (0 for in-bank cells)."""
    tot = state["rivsto"][0] + state["fldsto"][0] + state.get("levsto", np.zeros((1, N)))[0]
    fsm = fldstomax.reshape(L, N)
    flooded = tot > rivstomax
    scanned = np.sum(tot[None, :] > fsm, axis=0) + 1
    scanned = np.minimum(scanned, L)
    return float(np.mean(np.where(flooded, scanned, 0)))


# ------------------------------------------------------------------------------------- CPU arms
def cpu_run(cdir: str, spin: int, nsteps: int, seed: int, omp: bool = True, budget_s: float = 25.0):
    """Runs the oracle on the bench workload from the same initial state and forcing: `spin`
    untimed coupling steps, then up to `nsteps` timed ones (fewer if `budget_s` runs out).
    Returns (cell-substeps, seconds, threads, steps timed)."""
    from oracle import Oracle

    o = Oracle(cdir, omp=omp)
    gr = o.d("grarea")
    fields = runoff_fields(gr, spin + nsteps, seed)
    for k in range(spin):
        o.put_runoff(fields[k])
        o.advance()
    sub = 0
    done = 0
    t0 = time.perf_counter()
    for k in range(spin, spin + nsteps):
        o.put_runoff(fields[k])
        nt, _ = o.advance()
        sub += nt
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    return o.nseqall * sub, el, o.threads(), done


def reference_arm(args) -> int:
    """The reference algorithm's CPU implementation (the OpenMP oracle on every host core) on the
    same workload, forcing and timed window of coupling steps as the GPU arm."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    cdir = case_dir("cfg1")
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    os.environ.setdefault("OMP_PROC_BIND", "close")
    spin = SPINUP_STEPS + args.warmup
    cells, secs, threads, done = cpu_run(cdir, spin, args.steps, seed=1, omp=True, budget_s=150.0)
    v = cells / secs
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": done,
        "warmup": args.warmup, "ms_per_step": secs / max(done, 1) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded config-1 case in the reference's map formats)",
        "config": bench_config(1, args.warmup, args.steps),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "cpu_model": cpu_model(),
                         "sample": f"{done} consecutive coupling steps after {spin} untimed ones (the GPU arm's "
                                   f"timed window), OpenMP oracle on {threads} threads"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# -------------------------------------------------------------------------------------- GPU arm
def gpu_arm(args) -> int:
    import torch

    ws, rank, local = dist_env()
    if ws > 1:
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    torch.cuda.set_device(local)
    from cmf_b200 import HostModel, PhysicsGPU

    cdir = case_dir("cfg1")
    if ws > 1:
        dist.barrier()
    h = HostModel(cdir)
    M = args.members
    g = PhysicsGPU(h, nmembers=M, device=local, launch_mode=args.launch_mode, block_size=args.block_size)
    N = h.dims.nseqall
    gr = h.map("grarea")
    W, K = args.warmup, args.steps
    total = SPINUP_STEPS + W + K
    fields = np.stack([runoff_fields(gr, total, seed=1 + 1000 * rank + m) for m in range(M)], axis=1)  # [T][M][N]
    dev = torch.device("cuda", local)
    runoff_dev = torch.from_numpy(fields).to(dev)
    runoff_host = torch.from_numpy(fields).pin_memory()
    stride = M * N
    stream = torch.cuda.ExternalStream(g.stream, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device=dev)
    base = SPINUP_STEPS + W

    # spin-up and warm-up (device pipeline); the state at the start of the timed window is kept so
    # that the end-to-end run times the same window of coupling steps
    g.advance_device(base, runoff_dev.data_ptr(), stride)
    g.synchronize()
    snapshot = g.get_state()

    # ---- timed region: device-resident.  The clock sampler runs from half a second before it, while
    # the same window of coupling steps is replayed (untimed, from the saved state), so the clock
    # record holds samples under this load even though the timed region itself is short.
    clk = ClockSampler(local).__enter__()
    clk.wait_first()
    clk.mark_load()
    t_rep = time.perf_counter()
    while not args.no_replay and time.perf_counter() - t_rep < 0.5:
        g.set_state(snapshot)
        g.advance_device(K, runoff_dev.data_ptr() + base * stride * 8, stride)
        g.synchronize()
    g.set_state(snapshot)
    c0 = g.counters()
    s0 = g.nt_stats()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clk.mark_start()
    for k in range(K):
        with torch.cuda.stream(stream):
            flush.fill_(k)
            evs[k][0].record(stream)
        g.advance_device(1, runoff_dev.data_ptr() + (base + k) * stride * 8, stride)
        with torch.cuda.stream(stream):
            evs[k][1].record(stream)
    torch.cuda.synchronize()
    g.synchronize()
    clk.mark_end()
    clk.__exit__(None, None, None)
    ms = sum(a.elapsed_time(b) for a, b in evs)
    c1 = g.counters()
    s1 = g.nt_stats()
    member_sub = c1["member_substeps"] - c0["member_substeps"]
    loop_iters = c1["loop_iters"] - c0["loop_iters"]
    launches = g.launches_per_step() * K + g.launches_per_substep() * loop_iters
    hist = s1["hist"] - s0["hist"]
    secs = ms / 1e3
    if ws > 1:
        t = torch.tensor([secs], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        secs = float(t.item())
        tot = torch.tensor([float(member_sub)], device=dev, dtype=torch.float64)
        dist.all_reduce(tot, op=dist.ReduceOp.SUM)
        member_sub_all = tot.item()
    else:
        member_sub_all = member_sub
    value = N * member_sub_all / secs

    # ---- e2e through the public API with host buffers, the same window from the same state
    g.set_state(snapshot)
    # pipelined public API: the next step's runoff uploads from pinned host memory while a step
    # runs, and every finished step's averaged discharge reads back into pinned host memory while
    # the next one runs (two buffers, so a read-back never lands in the one the host reads)
    outs = [{"outflw_aavg": torch.zeros(M * N, dtype=torch.float64).pin_memory().numpy()} for _ in range(2)]
    rin = [runoff_host[base + k].numpy() for k in range(K)]
    io = g.pipeline(outs)            # the per-step calls with their ctypes arguments built once
    # untimed: two pipelined steps create the copy streams, pinned rings and staging buffers (a
    # one-time setup, like the context itself); then the saved state again
    for w in range(2):
        g.put_runoff_async(rin[w % K])
        io.advance()
        io.wait()
        io.read_back(w % 2)
        io.io_wait()
    g.set_state(snapshot)
    e2e_sub = 0
    budgets = []
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    # two steps in flight: step k+1 is already queued when the host waits for step k
    g.put_runoff_async(rin[0])
    io.advance()
    io.read_back(0)
    if K > 1:
        g.put_runoff_async(rin[1])
        io.advance()
    for k in range(K):
        nt = io.wait()               # step k
        io.io_wait()                 # step k's discharge is in the host buffer
        e2e_sub += int(nt.sum())
        budgets.append(io.budget(0))
        if k + 1 < K:
            io.read_back((k + 1) % 2)    # staged after step k+1, before step k+2
        if k + 2 < K:
            g.put_runoff_async(rin[k + 2])
            io.advance()
    e2e_secs = time.perf_counter() - t0
    if ws > 1:
        t = torch.tensor([e2e_secs], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_secs = float(t.item())
        tot = torch.tensor([float(e2e_sub)], device=dev, dtype=torch.float64)
        dist.all_reduce(tot, op=dist.ReduceOp.SUM)
        e2e_sub = tot.item()
    e2e_value = N * e2e_sub / e2e_secs

    # ---- roofline of the dominant kernel, timed live on the library's stream
    st = g.get_state()
    Lbar = mean_layers(st, h.map("fldstomax"), h.map("rivstomax"), N, h.dims.nlfp)
    E = int(h.map("i1upn").sum())
    P = g.P
    Lp = g.Lp
    nlev = int(np.sum(h.map("levbassto") < 1e17)) if h.opts.llevee else 0
    ndam = h.dims.ndam
    roof = roofline(g, N, E, Lbar, P, Lp, nlev, ndam, M, loop_iters, K, secs)

    # the one-member context is done: closed here, so that the 16-member and surrogate contexts
    # below each hold the hot-map L2 window in turn (one context holds it at a time)
    sched = g.schedule()
    g.close()

    # ---- 16 config-1 members on one context (the at-scale bandwidth, working set far above L2)
    wide = None
    if ws == 1 and not args.no_wide and M == 1:
        wide = members_line(h, dev, 16, fields[:, 0, :], base, min(K, 10), roof_args=(N, E, Lbar, P, Lp, nlev, ndam))

    sur = None
    if ws == 1 and not args.no_surrogate:
        from cmf_b200 import surrogate

        try:
            sur = surrogate.measure(h, dev, members=args.sur_members, days=args.sur_days,
                                    snapshot_weighting=args.sur_snapshots,
                                    trajectory_forcing=args.sur_traj_forcing or None)
        except Exception as e:       # reported, never silently replaced by another number
            sur = {"error": f"{type(e).__name__}: {e}"}
    out = 0
    if rank == 0:
        cpu = None
        if ws == 1 and not args.no_cpu:
            os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
            cells, csecs, threads, done = cpu_run(cdir, base, K, seed=1, omp=True, budget_s=20.0)
            cells1, csecs1, _, done1 = cpu_run(cdir, base, K, seed=1, omp=False, budget_s=10.0)
            cpu = {"value": cells / csecs, "unit": UNIT, "cores": threads, "kind": "port", "cpu_model": cpu_model(),
                   "sample": f"{done} consecutive coupling steps of the timed window (after {base} untimed ones) "
                             f"of the OpenMP oracle, {csecs:.1f} s on {threads} host threads",
                   "single_thread": {"value": cells1 / csecs1, "unit": UNIT, "cores": 1,
                                     "sample": f"{done1} coupling steps of the same window, serial oracle, {csecs1:.1f} s"}}
        # the loaded span: the untimed replay of the same coupling steps right before the timed
        # region plus the timed region itself (which alone lasts only tens of milliseconds)
        clocks = clk.summary(loaded=True)
        clocks["span"] = "replay of the timed steps (0.5 s) + timed region"
        clocks["timed_region"] = clk.summary()
        nthist = {str(k): int(v) for k, v in enumerate(hist) if v}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": K, "warmup": W,
            "ms_per_step": secs / K * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded config-1 case in the reference's map formats)",
            "config": bench_config(M, W, K),
            "details": {"parallelism": f"ensemble members sharded over {ws} GPU(s), no collective",
                        "l2": "256 MiB buffer written before every timed step", "nt_mean": member_sub / max(K * M, 1),
                        "nt_histogram": nthist, "nt_near_integer_steps": int(s1["near_boundary"] - s0["near_boundary"]),
                        "schedule": sched,
                        "launch": ("one CUDA graph per coupling step, device-side sub-step loop" if args.launch_mode == 0
                                   else "host-driven kernel launches")},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": M * N * 8,
                    "d2h_bytes_per_step": M * N * 8 + M * 160,
                    "window": "the same coupling steps as `value`, restarted from the saved state",
                    "host_buffers": "pinned (runoff in, averaged discharge out)",
                    "io": "pipelined, two steps in flight: the next steps' runoff uploads and the "
                          "finished step's discharge reads back while steps run (put_runoff_async / "
                          "advance_async / wait / get_diag_async / io_wait)"},
            "mass_balance": closure(budgets),
            "gpu_launches": int(launches),
            "roofline": roof,
            "members16": wide,
            "cpu_baseline": cpu,
            "clocks": clocks,
            "surrogate": sur,
        }
        print(json.dumps(line))
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    g.close()
    return out


def roofline(g, N, E, Lbar, P, Lp, nlev, ndam, M, loop_iters, K, secs) -> dict:
    """Dominant kernel's achieved bandwidth on algorithmic bytes (live CUDA-event timing on the
    library's stream) and the whole step's, on the fused minimum per cell-sub-step (316 + 16 L_bar
    B, plus 32 + 40 Lp per path, 80 per levee cell and 112 per dam)."""
    phases = g.time_phases(reps=10)
    pb = phase_bytes(N, E, Lbar, P, Lp, nlev, ndam, True)
    per_sub_ms = {k: phases[k] for k in ("k_flux", "k_rate", "k_store")}
    dominant = max(per_sub_ms, key=per_sub_ms.get)
    peaks = measured_peaks()
    achieved = pb[dominant] * M / (per_sub_ms[dominant] * 1e-3) / 1e9
    fused = fused_minimum_bytes(N, Lbar, P, Lp, nlev, ndam)
    step_gbs = fused * M * (loop_iters / max(K, 1)) / (secs / K) / 1e9
    return {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / peaks["hbm_gbs"], "traffic": None,
            "traffic_note": "not measured in this run (ncu summaries under profiles/)",
            "kernel": dominant, "peak_source": peaks["source"] + " (hbm_gbs, burst copy)",
            "algorithmic_bytes_per_launch": pb[dominant] * M,
            "kernel_ms": {k: round(v, 5) for k, v in phases.items()}, "L_bar": Lbar,
            "step_fused_minimum_bytes_per_substep": fused * M,
            "step_achieved_gbs": step_gbs, "step_frac": step_gbs / peaks["hbm_gbs"]}


def fused_minimum_bytes(N, Lbar, P, Lp, nlev, ndam) -> float:
    """Compulsory bytes of a fully fused sub-step: (316 + 16 L_bar) per cell, 32 + 40 Lp per
    bifurcation path, 80 per levee cell, 112 per dam (diagnostic accumulators not counted)."""
    return N * (316 + 16 * Lbar) + P * (32 + 40 * Lp) + nlev * 80 + ndam * 112


def members_line(h, dev, M, base_fields, base, K, roof_args) -> dict:
    """M config-1 members on one context, each member the bench forcing times a lognormal(0, 0.3)
    factor per cell: cell-substeps/s and the whole step's bandwidth on fused-minimum bytes."""
    import torch

    from cmf_b200 import PhysicsGPU

    N = h.dims.nseqall
    g = PhysicsGPU(h, nmembers=M, device=dev.index or 0)
    rng = np.random.default_rng(16)
    fac = np.exp(rng.normal(0.0, 0.3, size=(M, N)) - 0.045)
    T = base + K
    fields = torch.empty((T, M, N), dtype=torch.float64, device=dev)
    for k in range(T):
        fields[k] = torch.from_numpy(base_fields[k][None, :] * fac).to(dev)
    g.advance_device(base, fields.data_ptr(), M * N)
    g.synchronize()
    stream = torch.cuda.ExternalStream(g.stream, device=dev)
    c0 = g.counters()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    g.advance_device(K, fields.data_ptr() + base * M * N * 8, M * N)
    e1.record(stream)
    e1.synchronize()
    secs = e0.elapsed_time(e1) / 1e3
    c1 = g.counters()
    sub = c1["member_substeps"] - c0["member_substeps"]
    iters = c1["loop_iters"] - c0["loop_iters"]
    Nn, E, Lbar, P, Lp, nlev, ndam = roof_args
    fused = fused_minimum_bytes(Nn, Lbar, P, Lp, nlev, ndam)
    gbs = fused * sub / secs / 1e9
    peak = measured_peaks()["hbm_gbs"]
    sched = {k: v for k, v in g.schedule().items() if k != "kernels"}
    g.close()
    del fields
    torch.cuda.empty_cache()
    return {"members": M, "cell_substeps_per_s": N * sub / secs, "ms_per_step": secs / K * 1e3,
            "nt_mean": sub / (K * M), "step_achieved_gbs": gbs, "step_frac": gbs / peak,
            "l2": "working set far above L2 (no flush needed)", "steps": K, "schedule": sched}


# ------------------------------------------------------------------------- batched config 2
def cfg2_arm(args) -> int:
    """Config 2: `--members` runoff-perturbation members on 8 regional domains of uneven size
    (50k to 2M cells, config-1 laws), every coupling step one graph launch for all domains and
    members, each member with its own adaptive DT.  Forcing: the config-1 AR(1) field of each
    domain times a per-member lognormal(0, 0.3) factor field, spatially smoothed (bilinear
    upsampling of a 16x coarser Gaussian field), resident in HBM.  Under torchrun the domain x
    member units are bin-packed over the ranks by cells x expected NT (regions.pack_units); the
    total work is fixed (strong scaling) and each rank advances its units with one graph launch."""
    import datetime

    import torch

    from cmf_b200 import HostModel, PhysicsBatch, PhysicsGPU, regions, synth
    from cmf_b200 import emulator as E

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if ws > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    M, W, K = args.members, args.warmup, args.steps
    t_gen = time.perf_counter()
    specs = synth.spec_config2()
    if rank == 0:
        for sp in specs:
            d = os.path.join(CASE_CACHE, sp.name)
            if not os.path.exists(os.path.join(d, "input_cmf.nam")):
                synth.write_case(synth.make_case(sp), d + ".tmp")
                os.rename(d + ".tmp", d)
    if ws > 1:
        dist.barrier()
    hosts = [HostModel(os.path.join(CASE_CACHE, sp.name)) for sp in specs]
    t_gen = time.perf_counter() - t_gen
    nt_exp = [regions.expected_nt(h.map("nxtdst"), h.map("rivhgt"), h.dims.nseqriv, h.dt) for h in hosts]
    owned = regions.pack_units([h.dims.nseqall * n for h, n in zip(hosts, nt_exp)], M, ws)[rank]
    used, ctxs, views, facs, gens = [], [], [], [], []
    g = torch.Generator(device=dev).manual_seed(7)
    for k, h in enumerate(hosts):
        # every rank draws all M members' factor fields, so member m's forcing does not depend on
        # the rank count; a rank keeps the rows of the members it owns
        z = torch.randn(M, 1, h.ny // 16 + 2, h.nx // 16 + 2, generator=g, device=dev, dtype=torch.float64)
        if not owned[k]:
            continue
        z = torch.nn.functional.interpolate(z, size=(h.ny, h.nx), mode="bilinear", align_corners=False)[:, 0]
        z = z[:, torch.as_tensor(h.i1seqy - 1, device=dev), torch.as_tensor(h.i1seqx - 1, device=dev)]
        z = z / z.std(dim=1, keepdim=True)
        p = PhysicsGPU(h, nmembers=len(owned[k]), device=local)
        used.append(k)
        ctxs.append(p)
        views.append(E.Features(p, np.ones(p.N)).runoff_view())
        facs.append(torch.exp(0.3 * z[torch.as_tensor(owned[k], device=dev)] - 0.045))
        gens.append(synth.AR1GammaRunoff(p.N, 100 + k))
        del z
    batch = PhysicsBatch(ctxs) if ctxs else None
    stream = torch.cuda.ExternalStream(batch.stream, device=dev) if batch else torch.cuda.current_stream(dev)
    cur = torch.cuda.current_stream(dev)

    def put():
        for k, v, f, gen in zip(used, views, facs, gens):
            base = np.maximum((gen.next().astype(np.float64) * hosts[k].map("grarea")) / 86400000.0, 0.0)
            torch.mul(torch.from_numpy(base).to(dev)[None, :], f, out=v)
        cur.synchronize()

    for _ in range(SPINUP_STEPS + W):
        put()
        if batch:
            batch.launch()
            batch.synchronize()
    c0 = [c.counters() for c in ctxs]
    ms = 0.0
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for _ in range(K):
            put()
            ev[0].record(stream)
            if batch:
                batch.launch()
            ev[1].record(stream)
            ev[1].synchronize()
            ms += ev[0].elapsed_time(ev[1])
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    c1 = [c.counters() for c in ctxs]
    secs = ms / 1e3
    cells = 0
    abytes = 0.0
    nts = [0.0] * len(hosts)
    launches = 0
    for k, p, a, b in zip(used, ctxs, c0, c1):
        h = hosts[k]
        launches += p.launches_per_step() * K + p.launches_per_substep() * (b["loop_iters"] - a["loop_iters"])
        sub = b["member_substeps"] - a["member_substeps"]
        cells += h.dims.nseqall * sub
        nts[k] = sub / (K * p.M)
        nlev = int(np.sum(h.map("levbassto") < 1e17)) if h.opts.llevee else 0
        pb = phase_bytes(h.dims.nseqall, int(h.map("i1upn").sum()), 0.0, p.P, p.Lp, nlev, h.dims.ndam, True)
        abytes += sum(pb.values()) * sub
    if ws > 1:
        t = torch.tensor([secs], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        secs = float(t.item())
        tot = torch.tensor([float(cells), abytes], device=dev, dtype=torch.float64)
        dist.all_reduce(tot, op=dist.ReduceOp.SUM)
        cells, abytes = float(tot[0].item()), float(tot[1].item())
        # member-weighted mean NT per domain over the ranks holding it
        w = torch.tensor([nts[k] * len(owned[k]) for k in range(len(hosts))] + [len(ms_) for ms_ in owned],
                         device=dev, dtype=torch.float64)
        dist.all_reduce(w, op=dist.ReduceOp.SUM)
        nd = len(hosts)
        nts = [float(w[k].item() / w[nd + k].item()) if w[nd + k].item() else 0.0 for k in range(nd)]
    bsizes = [c.block_size for c in ctxs]
    if batch:
        batch.close()
    for c in ctxs:
        c.close()
    if rank != 0:
        if ws > 1:
            dist.destroy_process_group()
        return 0
    peaks = measured_peaks()
    value = cells / secs
    achieved = abytes / secs / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": K, "warmup": W,
        "ms_per_step": secs * 1e3 / K, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded config-2 domains in the reference's map formats)",
        "config": {"workload": "config2: 8 regional domains (config-1 laws), " +
                               ", ".join(str(h.dims.nseqall) for h in hosts) + " cells, "
                               f"{M} members each, one graph launch per coupling step per GPU",
                   "members": M, "cells_total": int(sum(h.dims.nseqall for h in hosts)),
                   "nt_mean_per_domain": [round(x, 2) for x in nts],
                   "nt_expected_per_domain": nt_exp,
                   "partition": "domain x member units bin-packed over the GPUs by cells x expected NT",
                   "units_per_gpu_rank0": [len(x) for x in owned],
                   "block_sizes_rank0": bsizes, "case_generation_s": round(t_gen, 1),
                   "l2": "working set far above L2 (no flush needed)"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"] / ws, "traffic": None, "kernel": "sub-step kernels (all)",
                     "peak_source": peaks["source"] + " (hbm_gbs, burst copy, per GPU)",
                     "note": "algorithmic bytes of k_flux+k_rate+k_store per member sub-step (L_bar taken as 0), "
                             "stage/CFL and control kernels not counted; achieved over all GPUs"},
        "clocks": clk.summary(),
        "gpu_launches": launches,
        "gpu_launches_scope": "rank 0",
    }
    print(json.dumps(line))
    if ws > 1:
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------------------ large single domain, config 4
def cfg4_arm(args) -> int:
    """Config 4: one ~6M-cell network (7200x3600 grid, config-1 laws, 100k bifurcation channels x 5
    levels, levees on 10% of cells, 10k dams).  (1) HBM-roofline sweep of the plain batched path
    over 1..M members (each member its own adaptive DT, one graph launch per coupling step), all
    sizes from the same spun-up state; (2) M members under the emulator with plain-solver judging
    against the plain path on the same ensemble (the surrogate measurement)."""
    import torch

    from cmf_b200 import HostModel, PhysicsGPU
    from cmf_b200 import emulator as E

    ws, rank, local = dist_env()
    if ws > 1 and rank != 0:
        return 0
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    t_gen = time.perf_counter()
    h = HostModel(case_dir("cfg4"))
    t_gen = time.perf_counter() - t_gen
    N, Mmax, W, K = h.dims.nseqall, args.members, args.warmup, args.steps
    spin = 12
    forcing = E.DeviceForcing(h, Mmax, spin + W + K, seed=41, device=dev, distinct=2)
    cur = torch.cuda.current_stream(dev)
    big = PhysicsGPU(h, nmembers=Mmax, device=local)
    view = E.Features(big, np.ones(N)).runoff_view()
    for k in range(spin):
        forcing.fill(k, view)
        cur.synchronize()
        big.advance_device(1, None, 0)
        big.synchronize()
    # mean floodplain layers the stage scheme scans (member 0 of the spun-up state, on the device)
    fe0 = E.Features(big, np.ones(N))
    tot = (E._raw_f64(fe0.mb.rivsto, N, dev) + E._raw_f64(fe0.mb.fldsto, N, dev) +
           (E._raw_f64(fe0.mb.levsto, N, dev) if fe0.mb.levsto else 0.0))
    L = h.dims.nlfp
    fsm = torch.as_tensor(h.map("fldstomax").reshape(L, N), device=dev)
    flooded = tot > torch.as_tensor(h.map("rivstomax"), device=dev)
    scanned = torch.clamp((tot[None, :] > fsm).sum(0) + 1, max=L)
    Lbar = float(torch.where(flooded, scanned, torch.zeros_like(scanned)).double().mean())
    del fsm, flooded, scanned, tot
    E_up = int(h.map("i1upn").sum())
    nlev = int(np.sum(h.map("levbassto") < 1e17)) if h.opts.llevee else 0
    pb = phase_bytes(N, E_up, Lbar, big.P, big.Lp, nlev, h.dims.ndam, True)
    peaks = measured_peaks()
    sweep = []
    top = None
    with ClockSampler(local) as clk:
        for M in sorted({m for m in (1, 2, 4, 8, 16, 32) if m <= Mmax} | {Mmax}, reverse=True):
            if M == Mmax:
                ctx = big
            else:
                ctx = PhysicsGPU(h, nmembers=M, device=local)
                for m in range(M):
                    E.check(E._emu_lib().cmf_gpu_ctx_copy_member(ctx.h, m, big.h, m), "copy_member")
            v = E.Features(ctx, np.ones(N)).runoff_view()
            stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
            for k in range(W):
                forcing.fill(spin + k, v)
                cur.synchronize()
                ctx.advance_device(1, None, 0)
            ctx.synchronize()
            c0 = ctx.counters()
            ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
            for k in range(K):
                forcing.fill(spin + W + k, v)
                cur.synchronize()
                ev[k][0].record(stream)
                ctx.advance_device(1, None, 0)
                ev[k][1].record(stream)
            ctx.synchronize()
            ms = sum(a.elapsed_time(b) for a, b in ev)
            c1 = ctx.counters()
            sub = c1["member_substeps"] - c0["member_substeps"]
            iters = c1["loop_iters"] - c0["loop_iters"]
            secs = ms / 1e3
            achieved = sum(pb.values()) * sub / secs / 1e9
            row = {"members": M, "cell_substeps_per_s": N * sub / secs, "ms_per_step": ms / K,
                   "nt_mean": sub / (K * M), "hbm_gbs": achieved, "hbm_frac": achieved / peaks["hbm_gbs"]}
            if M == Mmax:
                phases = ctx.time_phases(reps=3)
                kst = pb["k_store"] * M / (phases["k_store"] * 1e-3) / 1e9
                row["kernel_ms"] = {k: round(x, 4) for k, x in phases.items()}
                row["k_store_hbm_frac"] = kst / peaks["hbm_gbs"]
                top = dict(row, secs=secs, sub=sub, launches=3 * K + 3 * iters, kst=kst)
            sweep.append(row)
            if ctx is not big:
                ctx.close()
    big.close()
    del forcing
    torch.cuda.empty_cache()
    sur = None
    if not args.no_surrogate:
        from cmf_b200 import surrogate

        try:
            # the headline controller setting only: a 16-member judge context of this domain alone
            # would need about 29 GB next to the two 57 GB ensemble contexts
            sur = surrogate.measure(h, dev, members=Mmax, days=args.sur_days, forcing_distinct=2,
                                    snapshot_weighting=args.sur_snapshots,
                                    trajectory_forcing=args.sur_traj_forcing or None, pareto=())
        except Exception as e:       # reported, never silently replaced by another number
            sur = {"error": f"{type(e).__name__}: {e}"}
    line = {
        "metric": METRIC, "value": N * top["sub"] / top["secs"], "unit": UNIT, "n_gpus": 1, "steps": K, "warmup": W,
        "ms_per_step": top["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded config-4 case in the reference's map formats)",
        "config": {"workload": f"config4: {h.nx}x{h.ny} grid, {N} cells, {big.P} bifurcation x{big.Lp}, "
                               f"levees 10%, {h.dims.ndam} dams, {Mmax} members, hourly AR(1) forcing",
                   "members": Mmax, "nt_mean": top["nt_mean"], "L_bar": Lbar, "case_generation_s": round(t_gen, 1),
                   "l2": "working set far above L2 (no flush needed)",
                   "launch": "one CUDA graph per coupling step, device-side sub-step loop"},
        "roofline": {"bound": "hbm", "achieved": top["kst"], "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": top["kst"] / peaks["hbm_gbs"], "traffic": None, "kernel": "k_store",
                     "peak_source": peaks["source"] + " (hbm_gbs, burst copy)",
                     "algorithmic_bytes_per_launch": pb["k_store"] * Mmax, "kernel_ms": top["kernel_ms"],
                     "step_achieved_gbs": top["hbm_gbs"], "step_frac": top["hbm_frac"]},
        "sweep": sweep,
        "gpu_launches": int(top["launches"]),
        "clocks": clk.summary(),
        "surrogate": sur,
    }
    print(json.dumps(line))
    return 0


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--members", type=int, default=1)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-wide", action="store_true", help="skip the 16-member config-1 sub-line")
    ap.add_argument("--block-size", type=int, default=0,
                    help="threads per block of the phase kernels (0: the autotuner's choice)")
    ap.add_argument("--no-replay", action="store_true",
                    help="skip the untimed replay of the window that keeps the clock sampler under load "
                         "(for profiler runs, which count launches)")
    ap.add_argument("--no-surrogate", action="store_true",
                    help="skip the surrogate-assisted vs plain ensemble measurement")
    ap.add_argument("--sur-members", type=int, default=256)
    ap.add_argument("--sur-days", type=int, default=2)
    ap.add_argument("--sur-snapshots", default="uniform", choices=["uniform", "discharge"],
                    help="training snapshot cells: uniform, or in proportion to sqrt(discharge scale)")
    ap.add_argument("--sur-traj-forcing", type=int, default=0,
                    help="K > 0: build the training trajectories' forcing on the device from K distinct fields")
    ap.add_argument("--launch-mode", type=int, default=0, choices=[0, 1, 2],
                    help="0: CUDA graph with a device-side sub-step loop; 1: the same kernels as plain "
                         "launches from a host loop (what ncu can profile kernel by kernel)")
    ap.add_argument("--workload", default="cfg1", choices=["cfg1", "cfg2", "cfg4"],
                    help="cfg1: the config-1 network (default); cfg2: the batched uneven multi-domain ensemble; "
                         "cfg4: the ~6M-cell single domain (plain member sweep + surrogate ensemble)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return reference_arm(args)
    if args.workload == "cfg2":
        if args.members == 1:
            args.members = 64
        return cfg2_arm(args)
    if args.workload == "cfg4":
        if args.members == 1:
            args.members = 32
        return cfg4_arm(args)
    return gpu_arm(args)


if __name__ == "__main__":
    sys.exit(main())
