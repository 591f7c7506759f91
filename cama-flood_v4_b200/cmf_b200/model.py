"""Host-side mirror of the reference driver interface for the GPU physics step.

``HostModel`` plays CMF_DRV_INIT (src/cmf_drv_control_mod.F90:149-298) for a case written in the
reference's file formats; ``PhysicsGPU`` is the GPU switch behind CMF_DRV_ADVANCE: each
``advance()`` is one CMF_PHYSICS_ADVANCE (src/cmf_ctrl_physics_mod.F90:21-153) for every member.
Errors surface as RuntimeError carrying the library's status and message; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import check


def _as_np(ptr, n, dtype):
    if not ptr or n <= 0:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,))


class HostModel:
    """Stand-alone host: reads input_cmf.nam, diminfo and the binary maps, runs the init chain."""

    def __init__(self, casedir: str, nml: str = "input_cmf.nam"):
        self.lib = _abi.load()
        h = C.c_void_p()
        check(self.lib.cmf_host_load(casedir.encode(), nml.encode(), C.byref(h)), "cmf_host_load")
        self.h = h
        self.dims = _abi.Dims()
        self.params = _abi.Params()
        self.maps = _abi.MapPtrs()
        self.opts = _abi.Opts()
        dt = C.c_double()
        check(self.lib.cmf_host_describe(self.h, C.byref(self.dims), C.byref(self.params), C.byref(self.maps),
                                         C.byref(self.opts), C.byref(dt)), "cmf_host_describe")
        self.dt = dt.value
        self._state = _abi.StatePtrs()
        check(self.lib.cmf_host_state(self.h, C.byref(self._state)), "cmf_host_state")
        nx, ny = C.c_int32(), C.c_int32()
        self.i1seqx = np.zeros(self.dims.nseqmax, dtype=np.int32)
        self.i1seqy = np.zeros(self.dims.nseqmax, dtype=np.int32)
        check(self.lib.cmf_host_grid(self.h, C.byref(nx), C.byref(ny),
                                     self.i1seqx.ctypes.data_as(_abi.i32p), self.i1seqy.ctypes.data_as(_abi.i32p)),
              "cmf_host_grid")
        self.nx, self.ny = nx.value, ny.value
        self.drofunit = float(self.lib.cmf_host_drofunit(self.h))

    @property
    def nseq(self) -> int:
        return self.dims.nseqall

    def _len(self, name: str) -> int:
        d = self.dims
        N, L = d.nseqmax, d.nlfp
        P, Lp = d.npthout, d.npthlev
        table = {
            "i1upst": N * d.upnmax, "fldstomax": N * L, "fldgrd": N * L, "fldhgt": N * L,
            "pth_upst": P, "pth_down": P, "pth_dst": P, "pth_elv": P * Lp, "pth_wth": P * Lp, "pth_man": Lp,
            "i1p_out": N * d.onmax, "i1p_inf": N * d.inmax,
            "damseq": d.ndam, "damstat": d.ndam,
        }
        if name.startswith("dam_"):
            return d.ndam
        return table.get(name, N)

    def map(self, name: str) -> np.ndarray:
        """Copy of one static map array of the boundary (Fortran layout, 1-based index values)."""
        ptr = getattr(self.maps, name)
        dtype = np.int32 if dict(_abi.MAP_FIELDS)[name] is _abi.i32p else np.float64
        return _as_np(ptr, self._len(name), dtype).copy()

    def initial_state(self) -> dict:
        d = self.dims
        out = {}
        for n in _abi.STATE_FIELDS:
            ln = d.npthout * d.npthlev if n.startswith("pthflw") else d.nseqmax
            out[n] = _as_np(getattr(self._state, n), ln, np.float64).copy()
        return out

    def conv_resol(self, runoff_map: np.ndarray) -> np.ndarray:
        """CONV_RESOL: runoff map [mm/dt as DROFUNIT says] -> D2RUNOFF [m3/s]."""
        a = np.ascontiguousarray(runoff_map, dtype=np.float64).ravel()
        assert a.size == self.nx * self.ny
        out = np.zeros(self.dims.nseqmax)
        check(self.lib.cmf_host_conv_resol(self.h, a.ctypes.data_as(_abi.f64p), out.ctypes.data_as(_abi.f64p)),
              "cmf_host_conv_resol")
        return out

    def runoff_from_cells(self, mm_per_day_cells: np.ndarray) -> np.ndarray:
        """Per-sequence-cell runoff [mm/day] -> m3/s with CONV_RESOL's arithmetic."""
        gr = self.map("grarea")
        v = np.asarray(mm_per_day_cells, dtype=np.float64)
        return np.maximum((v * gr) / 86400000.0, 0.0)

    def _state_struct(self, state: dict, keep: list):
        sp = _abi.StatePtrs()
        for n in _abi.STATE_FIELDS:
            if n in state and state[n] is not None:
                a = state[n]
                if a.dtype != np.float64 or not a.flags.c_contiguous:
                    raise ValueError(n)
                keep.append(a)
                setattr(sp, n, a.ctypes.data_as(_abi.f64p))
        return sp

    def write_restart(self, path: str, state: dict, dbl: bool = True, stoonly: bool = False) -> None:
        """CMF_RESTART_WRITE's binary file (src/cmf_ctrl_restart_mod.F90:389-482) from one member's
        state arrays (keys of STATE_FIELDS, sequence order)."""
        keep: list = []
        st = {k: np.ascontiguousarray(v, dtype=np.float64).ravel() for k, v in state.items()}
        sp = self._state_struct(st, keep)
        check(self.lib.cmf_host_write_restart(self.h, C.byref(sp), path.encode(), int(dbl), int(stoonly)),
              "cmf_host_write_restart")

    def read_restart(self, path: str, dbl: bool = True, stoonly: bool = False) -> dict:
        """CMF_RESTART_INIT's binary read (src/cmf_ctrl_restart_mod.F90:91-204) -> one member's state."""
        d = self.dims
        st = {n: np.zeros(d.npthout * d.npthlev if n.startswith("pthflw") else d.nseqmax) for n in _abi.STATE_FIELDS}
        keep: list = []
        sp = self._state_struct(st, keep)
        check(self.lib.cmf_host_read_restart(self.h, C.byref(sp), path.encode(), int(dbl), int(stoonly)),
              "cmf_host_read_restart")
        return st

    def read_inpmat(self, path: str, inpn: int):
        """CMF_INPMAT_INIT_BIN: (inpx, inpy, inpa) in sequence order, [INPN][NSEQMAX] each."""
        N = self.dims.nseqmax
        ix = np.zeros(inpn * N, dtype=np.int32)
        iy = np.zeros(inpn * N, dtype=np.int32)
        ia = np.zeros(inpn * N)
        check(self.lib.cmf_host_read_inpmat(self.h, path.encode(), inpn, ix.ctypes.data_as(_abi.i32p),
                                            iy.ctypes.data_as(_abi.i32p), ia.ctypes.data_as(_abi.f64p)), "read_inpmat")
        return ix.reshape(inpn, N), iy.reshape(inpn, N), ia.reshape(inpn, N)

    def map_to_vec(self, map2d: np.ndarray) -> np.ndarray:
        """mapR2vecD: float32 NX x NY map (e.g. a sea-level record) -> sequence-order float64."""
        a = np.ascontiguousarray(map2d, dtype=np.float32).ravel()
        assert a.size == self.nx * self.ny
        out = np.zeros(self.dims.nseqmax)
        check(self.lib.cmf_host_map_to_vec(self.h, a.ctypes.data_as(C.POINTER(C.c_float)), out.ctypes.data_as(_abi.f64p)),
              "cmf_host_map_to_vec")
        return out

    def grid_to_seq(self, grid: np.ndarray) -> np.ndarray:
        g = np.asarray(grid).reshape(self.ny, self.nx)
        return g[self.i1seqy - 1, self.i1seqx - 1]

    def close(self) -> None:
        if self.h:
            self.lib.cmf_host_free(self.h)
            self.h = None


class PhysicsGPU:
    """A GPU context running ``nmembers`` members of the host model's network."""

    def __init__(self, host: HostModel, nmembers: int = 1, ldiag: bool = True, launch_mode: int = 0,
                 device: int = 0, block_size: int = 0, opts_override: dict | None = None, ldiag_output: bool = False):
        self.lib = _abi.load()
        self.host = host
        dims = _abi.Dims.from_buffer_copy(host.dims)
        dims.nmembers = nmembers
        opts = _abi.Opts.from_buffer_copy(host.opts)
        opts.ldiag = int(ldiag)
        opts.launch_mode = launch_mode
        opts.device = device
        opts.block_size = block_size
        opts.ldiag_output = int(ldiag_output)
        for k, v in (opts_override or {}).items():
            setattr(opts, k, int(v))
        self.dims, self.opts = dims, opts
        self.M = nmembers
        self.N = dims.nseqall
        self.P = dims.npthout if opts.lpthout else 0
        self.Lp = dims.npthlev if opts.lpthout else 0
        h = C.c_void_p()
        check(self.lib.cmf_gpu_create(C.byref(dims), C.byref(host.params), C.byref(host.maps), C.byref(opts),
                                      C.byref(h)), "cmf_gpu_create")
        self.h = h
        st = host.initial_state()
        self.set_state({k: np.tile(v, nmembers) for k, v in st.items()})

    # ---- state ------------------------------------------------------------------------------
    def _state_sizes(self, name: str) -> int:
        if name.startswith("pthflw"):
            return self.M * max(self.host.dims.npthout * self.host.dims.npthlev, 1)
        return self.M * self.N

    def set_state(self, state: dict) -> None:
        sp = _abi.StatePtrs()
        keep = []
        for n in _abi.STATE_FIELDS:
            if n in state and state[n] is not None:
                a = np.ascontiguousarray(state[n], dtype=np.float64).ravel()
                if a.size != self._state_sizes(n):
                    raise ValueError(f"{n}: expected {self._state_sizes(n)} values, got {a.size}")
                keep.append(a)
                setattr(sp, n, a.ctypes.data_as(_abi.f64p))
        check(self.lib.cmf_gpu_ctx_set_state(self.h, C.byref(sp)), "set_state")

    def get_state(self) -> dict:
        sp = _abi.StatePtrs()
        out = {}
        for n in _abi.STATE_FIELDS:
            a = np.zeros(self._state_sizes(n))
            out[n] = a
            setattr(sp, n, a.ctypes.data_as(_abi.f64p))
        check(self.lib.cmf_gpu_ctx_get_state(self.h, C.byref(sp)), "get_state")
        return {k: v.reshape(self.M, -1) for k, v in out.items()}

    def write_restart(self, path: str, member: int = 0, dbl: bool = True, stoonly: bool = False) -> None:
        """Device state of one member -> the reference's binary restart file (and .pth)."""
        st = self.get_state()
        self.host.write_restart(path, {k: v[member] for k, v in st.items()}, dbl=dbl, stoonly=stoonly)

    def read_restart(self, path: str, dbl: bool = True, stoonly: bool = False, members=None) -> None:
        """Restart file -> the device state of the given members (all by default).  A storage-only
        restart then reconstructs the previous-step flows with calc_outpre(), as CMF_DRV_INIT does."""
        one = self.host.read_restart(path, dbl=dbl, stoonly=stoonly)
        members = range(self.M) if members is None else list(members)
        st = self.get_state()
        for k, v in one.items():
            for m in members:
                st[k][m] = v
        self.set_state(st)
        if stoonly:
            self.calc_outpre()

    def set_runoff_map(self, inpmat=None) -> None:
        """Device runoff interpolation: inpmat = (nxin, nyin, inpx, inpy, inpa) -> ROFF_INTERP; None ->
        CONV_RESOL on the map grid."""
        keep = []
        if inpmat is None:
            nxin, nyin, inpn = self.host.nx, self.host.ny, 1
            ix, iy, ia = self.host.i1seqx, self.host.i1seqy, None
            lint = 0
        else:
            nxin, nyin, ix, iy, ia = inpmat
            ix = np.ascontiguousarray(ix, dtype=np.int32).ravel()
            iy = np.ascontiguousarray(iy, dtype=np.int32).ravel()
            ia = np.ascontiguousarray(ia, dtype=np.float64).ravel()
            inpn = ix.size // self.N
            lint = 1
        keep += [ix, iy, ia]
        self._rmap = (nxin, nyin)
        check(self.lib.cmf_gpu_ctx_set_runoff_map(self.h, lint, nxin, nyin, inpn, ix.ctypes.data_as(_abi.i32p),
                                                  iy.ctypes.data_as(_abi.i32p),
                                                  None if ia is None else ia.ctypes.data_as(_abi.f64p),
                                                  float(self.host.drofunit)), "set_runoff_map")

    def put_runoff_grid(self, grid, clean: bool = False) -> None:
        """Runoff fields [nmembers, NYIN, NXIN] (numpy fp32/fp64 on the host, or a CUDA tensor) ->
        D2RUNOFF of every member through the device interpolation."""
        if hasattr(grid, "data_ptr"):
            import torch

            is_float = grid.dtype == torch.float32
            torch.cuda.current_stream(grid.device).synchronize()
            check(self.lib.cmf_gpu_ctx_put_runoff_grid(self.h, C.c_void_p(grid.data_ptr()), int(is_float), 1, int(clean)),
                  "put_runoff_grid")
            return
        a = np.ascontiguousarray(grid)
        if a.dtype not in (np.float32, np.float64):
            a = a.astype(np.float64)
        if a.size != self.M * self._rmap[0] * self._rmap[1]:
            raise ValueError("runoff grid must hold nmembers * NXIN * NYIN values")
        check(self.lib.cmf_gpu_ctx_put_runoff_grid(self.h, a.ctypes.data_as(C.c_void_p), int(a.dtype == np.float32), 0,
                                                   int(clean)), "put_runoff_grid")

    def calc_outpre(self) -> None:
        """Stage scheme + CMF_CALC_OUTPRE on the device (storage-only restart)."""
        check(self.lib.cmf_gpu_ctx_calc_outpre(self.h), "calc_outpre")

    def update_boundary(self, sealev: np.ndarray | None = None, meansl: np.ndarray | None = None) -> None:
        """CMF_BOUNDARY_UPDATE: D2DWNELV = D2ELEVTN (+ meansl) (+ sealev), sequence-order arrays."""
        keep = []
        ptrs = []
        for a in (sealev, meansl):
            if a is None:
                ptrs.append(None)
            else:
                v = np.ascontiguousarray(a, dtype=np.float64).ravel()
                if v.size != self.N:
                    raise ValueError("boundary arrays hold NSEQALL values")
                keep.append(v)
                ptrs.append(v.ctypes.data_as(_abi.f64p))
        check(self.lib.cmf_gpu_ctx_update_boundary(self.h, ptrs[0], ptrs[1]), "update_boundary")

    def put_runoff(self, runoff: np.ndarray) -> None:
        a = np.ascontiguousarray(runoff, dtype=np.float64).ravel()
        if a.size != self.M * self.N:
            raise ValueError("runoff must hold nmembers * NSEQALL values")
        check(self.lib.cmf_gpu_ctx_put_runoff(self.h, a.ctypes.data_as(_abi.f64p), None), "put_runoff")

    def advance(self, dt_def: float | None = None):
        dt_def = self.host.dt if dt_def is None else dt_def
        nt = np.zeros(self.M, dtype=np.int32)
        dt = np.zeros(self.M)
        b = (_abi.Budget * self.M)()
        check(self.lib.cmf_gpu_ctx_physics_advance(self.h, dt_def, nt.ctypes.data_as(_abi.i32p),
                                                   dt.ctypes.data_as(_abi.f64p), b), "physics_advance")
        budgets = [{f: getattr(b[m], f) for f in _abi.BUDGET_FIELDS} for m in range(self.M)]
        return nt, dt, budgets

    def stage(self, dt_def: float | None = None) -> np.ndarray:
        dt_def = self.host.dt if dt_def is None else dt_def
        out = np.zeros(self.M)
        check(self.lib.cmf_gpu_ctx_stage(self.h, dt_def, out.ctypes.data_as(_abi.f64p)), "stage")
        return out

    def substeps(self, dt_min_global: float, dt_def: float | None = None):
        dt_def = self.host.dt if dt_def is None else dt_def
        nt = np.zeros(self.M, dtype=np.int32)
        dt = np.zeros(self.M)
        b = (_abi.Budget * self.M)()
        check(self.lib.cmf_gpu_ctx_substeps(self.h, dt_def, dt_min_global, nt.ctypes.data_as(_abi.i32p),
                                            dt.ctypes.data_as(_abi.f64p), b), "substeps")
        return nt, dt, [{f: getattr(b[m], f) for f in _abi.BUDGET_FIELDS} for m in range(self.M)]

    def advance_device(self, ksteps: int, runoff_dev_ptr: int | None, stride: int, dt_def: float | None = None) -> None:
        dt_def = self.host.dt if dt_def is None else dt_def
        check(self.lib.cmf_gpu_ctx_advance_device(self.h, dt_def, ksteps, C.c_void_p(runoff_dev_ptr or 0), stride),
              "advance_device")

    def synchronize(self) -> None:
        check(self.lib.cmf_gpu_ctx_synchronize(self.h), "synchronize")

    def last_nt(self):
        nt = np.zeros(self.M, dtype=np.int32)
        dt = np.zeros(self.M)
        check(self.lib.cmf_gpu_ctx_last_nt(self.h, nt.ctypes.data_as(_abi.i32p), dt.ctypes.data_as(_abi.f64p)), "last_nt")
        return nt, dt

    def counters(self):
        a, b, c = C.c_int64(), C.c_int64(), C.c_int64()
        check(self.lib.cmf_gpu_ctx_counters(self.h, C.byref(a), C.byref(b), C.byref(c)), "counters")
        return {"member_substeps": a.value, "loop_iters": b.value, "outer_steps": c.value}

    def nt_stats(self, nbins: int = 64) -> dict:
        """NT histogram over (outer step, member) pairs since creation, and how many of them had
        DT_DEF/DT_MIN - 0.01 within 1e-12 (relative) of an integer (NT hangs on DT_MIN's last bits)."""
        near = C.c_int64()
        hist = np.zeros(nbins, dtype=np.int64)
        check(self.lib.cmf_gpu_ctx_nt_stats(self.h, C.byref(near), hist.ctypes.data_as(C.POINTER(C.c_int64)), nbins),
              "nt_stats")
        return {"near_boundary": near.value, "hist": hist}

    def time_phases(self, reps: int = 10, dt_def: float | None = None) -> dict:
        dt_def = self.host.dt if dt_def is None else dt_def
        ms = np.zeros(6)
        check(self.lib.cmf_gpu_ctx_time_phases(self.h, dt_def, reps, ms.ctypes.data_as(_abi.f64p)), "time_phases")
        return dict(zip(["k_stage", "k_ntdt", "k_flux", "k_rate", "k_store", "k_budget"], ms.tolist()))

    @property
    def stream(self) -> int:
        return int(self.lib.cmf_gpu_ctx_stream(self.h) or 0)

    @property
    def kernel_launches(self) -> int:
        return int(self.lib.cmf_gpu_ctx_kernel_launches(self.h))

    @property
    def block_size(self) -> int:
        return int(self.lib.cmf_gpu_ctx_block_size(self.h))

    @property
    def launch_mode(self) -> int:
        """0: graph of phase kernels, 1: host-driven phase kernels, 2: persistent kernel."""
        return int(self.lib.cmf_gpu_ctx_launch_mode(self.h))

    def schedule(self) -> dict:
        """The launch schedule the context runs (chosen by the online autotuner unless fixed)."""
        q = _abi.Schedule()
        check(self.lib.cmf_gpu_ctx_get_schedule(self.h, C.byref(q)), "get_schedule")
        d = {f: getattr(q, f) for f, _ in _abi.Schedule._fields_}
        d["kernels"] = ("one persistent cooperative kernel per coupling step (grid barriers between phases, "
                        "tiles of 256 cells interleaved over the CTAs)" if q.mode == 2 else
                        "graph: stage, NT/DT, {flux, rate, store} x NT, budget")
        return d

    def set_schedule(self, mode: int = 0, flux_block: int = 128, rate_block: int = 128, store_block: int = 128,
                     profile: int = 1) -> None:
        q = _abi.Schedule(mode=mode, flux_block=flux_block, rate_block=rate_block, store_block=store_block,
                          profile=profile)
        check(self.lib.cmf_gpu_ctx_set_schedule(self.h, C.byref(q)), "set_schedule")

    def launches_per_step(self) -> int:
        """Kernel launches per outer step outside the sub-step loop."""
        return 1 if self.launch_mode == 2 else 3

    def launches_per_substep(self) -> int:
        return 0 if self.launch_mode == 2 else 3

    def persist_selftest(self, wait_ns: int = 2_000_000) -> int:
        """Status of the persistent kernel's bounded-wait check (CMF_E_BARRIER = 5 when it works)."""
        return int(self.lib.cmf_gpu_ctx_persist_selftest(self.h, int(wait_ns)))

    def diag_len(self, name: str) -> int:
        """Elements of the named diagnostic over all members (the host array's size)."""
        MP = self.M * max(self.P, 1)
        if name in ("pthflwsum", "pthflwsum_aavg"):
            return MP
        if name == "pthflw_aavg":
            return MP * max(self.Lp, 1)
        return self.M * self.N

    def _diag_ptrs(self, out: dict) -> "_abi.DiagPtrs":
        """Pointer struct for named float64 host arrays, each checked for name, type and size."""
        dp = _abi.DiagPtrs()
        for n, a in out.items():
            if n not in _abi.DIAG_FIELDS or a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError(n)
            if a.size < self.diag_len(n):
                raise ValueError(f"{n}: {a.size} elements, {self.diag_len(n)} needed")
            setattr(dp, n, a.ctypes.data_as(_abi.f64p))
        return dp

    def get_diag(self) -> dict:
        dp = _abi.DiagPtrs()
        out = {}
        for n in _abi.DIAG_FIELDS:
            a = np.zeros(self.diag_len(n))
            out[n] = a
            setattr(dp, n, a.ctypes.data_as(_abi.f64p))
        check(self.lib.cmf_gpu_ctx_get_diag(self.h, C.byref(dp)), "get_diag")
        return {k: v.reshape(self.M, -1) for k, v in out.items()}

    def diag_output(self, op: str) -> None:
        """CMF_DIAG_GETAVE_OUTPUT ("getave") or CMF_DIAG_RESET_OUTPUT ("reset") on the device; the
        AVEMAX step runs inside every advance() when the context was made with ldiag_output."""
        check(self.lib.cmf_gpu_ctx_diag_output(self.h, {"reset": 0, "getave": 2}[op]), "diag_output")

    def get_diag_output(self) -> dict:
        """The output-interval averages/maxima (D2*_oAVG, D2*_oMAX, D1PTHFLW_oAVG) and NADD_out."""
        dp = _abi.DiagOutPtrs()
        out = {}
        for n in _abi.DIAG_OUT_FIELDS:
            ln = self.M if n == "nadd_out" else (self.M * max(self.P * self.Lp, 1) if n == "pthflw_oavg" else self.M * self.N)
            a = np.zeros(ln)
            out[n] = a
            setattr(dp, n, a.ctypes.data_as(_abi.f64p))
        check(self.lib.cmf_gpu_ctx_get_diag_output(self.h, C.byref(dp)), "get_diag_output")
        return {k: v.reshape(self.M, -1) for k, v in out.items()}

    # ---- pipelined host I/O: the next step's runoff uploads while a step runs, and a finished
    # step's diagnostics read back while the next one runs (host arrays should be pinned)
    def put_runoff_async(self, runoff: np.ndarray) -> None:
        """Stages D2RUNOFF of the next outer step (float64, nmembers * NSEQALL, C-contiguous; the
        array must stay alive and unchanged until the next advance has been launched)."""
        if runoff.dtype != np.float64 or not runoff.flags.c_contiguous or runoff.size != self.M * self.N:
            raise ValueError("runoff must be a C-contiguous float64 array of nmembers * NSEQALL values")
        check(self.lib.cmf_gpu_ctx_put_runoff_async(self.h, runoff.ctypes.data_as(_abi.f64p)), "put_runoff_async")

    def advance_async(self, dt_def: float | None = None) -> None:
        dt_def = self.host.dt if dt_def is None else dt_def
        check(self.lib.cmf_gpu_ctx_advance_async(self.h, dt_def), "advance_async")

    def wait(self):
        """Finishes the step advance_async launched: (nt, dt, budgets) like advance()."""
        nt = np.zeros(self.M, dtype=np.int32)
        dt = np.zeros(self.M)
        b = (_abi.Budget * self.M)()
        check(self.lib.cmf_gpu_ctx_wait(self.h, nt.ctypes.data_as(_abi.i32p), dt.ctypes.data_as(_abi.f64p), b), "wait")
        return nt, dt, [{f: getattr(b[m], f) for f in _abi.BUDGET_FIELDS} for m in range(self.M)]

    def get_diag_fields_async(self, out: dict) -> None:
        """Starts the read-back of the named diagnostics into the caller's float64 arrays (they
        land by io_wait(); the arrays must stay alive until then)."""
        dp = self._diag_ptrs(out)
        check(self.lib.cmf_gpu_ctx_get_diag_async(self.h, C.byref(dp)), "get_diag_async")

    def io_wait(self) -> None:
        check(self.lib.cmf_gpu_ctx_io_wait(self.h), "io_wait")

    def pipeline(self, outs: list) -> "Pipeline":
        """The pipelined calls of a step loop with their ctypes arguments built once: `outs` are
        dicts of float64 host arrays (named diagnostics), one dict per read-back buffer."""
        return Pipeline(self, outs)

    def get_diag_fields(self, out: dict) -> dict:
        """Copies only the named diagnostics into the caller's float64 arrays (others skipped)."""
        dp = self._diag_ptrs(out)
        check(self.lib.cmf_gpu_ctx_get_diag(self.h, C.byref(dp)), "get_diag")
        return out

    def close(self) -> None:
        if self.h:
            self.lib.cmf_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PhysicsBatch:
    """Contexts of several domains (each with its own members) advanced by one graph launch per
    coupling step; every domain and member keeps its own adaptive DT."""

    def __init__(self, contexts: list):
        self.lib = _abi.load()
        self.ctx = list(contexts)
        arr = (C.c_void_p * len(self.ctx))(*[c.h.value if isinstance(c.h, C.c_void_p) else c.h for c in self.ctx])
        h = C.c_void_p()
        check(self.lib.cmf_gpu_batch_create(arr, len(self.ctx), C.byref(h)), "cmf_gpu_batch_create")
        self.h = h
        self.members = sum(c.M for c in self.ctx)

    def launch(self, dt_def: float | None = None) -> None:
        dt_def = self.ctx[0].host.dt if dt_def is None else dt_def
        check(self.lib.cmf_gpu_batch_launch(self.h, dt_def), "batch_launch")

    def advance(self, dt_def: float | None = None):
        """One coupling step of every domain; returns per-domain lists (nt, dt) like PhysicsGPU.advance."""
        dt_def = self.ctx[0].host.dt if dt_def is None else dt_def
        nt = np.zeros(self.members, dtype=np.int32)
        dt = np.zeros(self.members)
        b = (_abi.Budget * self.members)()
        check(self.lib.cmf_gpu_batch_advance(self.h, dt_def, nt.ctypes.data_as(_abi.i32p), dt.ctypes.data_as(_abi.f64p), b),
              "batch_advance")
        out, off = [], 0
        for c in self.ctx:
            out.append((nt[off:off + c.M], dt[off:off + c.M],
                        [{f: getattr(b[off + m], f) for f in _abi.BUDGET_FIELDS} for m in range(c.M)]))
            off += c.M
        return out

    def synchronize(self) -> None:
        check(self.lib.cmf_gpu_batch_synchronize(self.h), "batch_synchronize")

    @property
    def stream(self) -> int:
        return self.lib.cmf_gpu_batch_stream(self.h)

    def close(self) -> None:
        if self.h:
            self.lib.cmf_gpu_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Pipeline:
    """Per-step calls of a pipelined loop (advance_async / wait / get_diag_async / io_wait) with
    their argument structs prebuilt, so that the host's part of the gap between two steps is a few
    C calls."""

    def __init__(self, g: PhysicsGPU, outs: list):
        self.g, self.lib, self.h, self.dt = g, g.lib, g.h, g.host.dt
        self.nt = np.zeros(g.M, dtype=np.int32)
        self.dtv = np.zeros(g.M)
        self.b = (_abi.Budget * g.M)()
        self._nt_p, self._dt_p = self.nt.ctypes.data_as(_abi.i32p), self.dtv.ctypes.data_as(_abi.f64p)
        self.outs = outs
        self.dps = [g._diag_ptrs(out) for out in outs]

    def advance(self) -> None:
        check(self.lib.cmf_gpu_ctx_advance_async(self.h, self.dt), "advance_async")

    def wait(self) -> np.ndarray:
        """Finishes the launched step; returns NT per member (DT in .dtv, budgets via budget())."""
        check(self.lib.cmf_gpu_ctx_wait(self.h, self._nt_p, self._dt_p, self.b), "wait")
        return self.nt

    def budget(self, m: int) -> dict:
        return {f: getattr(self.b[m], f) for f in _abi.BUDGET_FIELDS}

    def read_back(self, slot: int) -> None:
        check(self.lib.cmf_gpu_ctx_get_diag_async(self.h, C.byref(self.dps[slot])), "get_diag_async")

    def io_wait(self) -> None:
        check(self.lib.cmf_gpu_ctx_io_wait(self.h), "io_wait")
