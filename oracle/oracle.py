"""ctypes wrapper of the CPU oracle (cmf_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
and reference arms as the checker.  The product never imports this module.

Parity is unpinned: the reference (Fortran 90) cannot be compiled on this machine and ships no
golden vectors for the physics step; see the header of cmf_oracle.c.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS: dict = {}


def build() -> None:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _lib(omp: bool = False):
    key = "omp" if omp else "serial"
    if key in _LIBS:
        return _LIBS[key]
    path = os.path.join(_HERE, "_build", "libcmf_oracle_omp.so" if omp else "libcmf_oracle.so")
    if not os.path.exists(path):
        build()
    lib = C.CDLL(path)
    lib.orc_create.restype = C.c_void_p
    lib.orc_create.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.c_int]
    lib.orc_physics_advance.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)]
    lib.orc_physics_advance.restype = C.c_int
    lib.orc_put_runoff_vec.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    lib.orc_put_runoff_map.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    lib.orc_dims.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
    lib.orc_budget.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    lib.orc_darray.restype = C.POINTER(C.c_double)
    lib.orc_darray.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_int)]
    lib.orc_iarray.restype = C.POINTER(C.c_int)
    lib.orc_iarray.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_int)]
    lib.orc_threads.restype = C.c_int
    lib.orc_stage.restype = C.c_double
    lib.orc_stage.argtypes = [C.c_void_p]
    lib.orc_substeps.argtypes = [C.c_void_p, C.c_double, C.POINTER(C.c_int), C.POINTER(C.c_double)]
    lib.orc_write_restart.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.c_int]
    lib.orc_read_restart.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.c_int]
    lib.orc_physics_fldstg.argtypes = [C.c_void_p]
    lib.orc_calc_outpre.argtypes = [C.c_void_p]
    lib.orc_forcing_clean.argtypes = [C.POINTER(C.c_double), C.c_size_t]
    lib.orc_roff_interp.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int),
                                    C.POINTER(C.c_int), C.POINTER(C.c_double)]
    lib.orc_update_boundary.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.orc_diag_output.argtypes = [C.c_void_p, C.c_int]
    lib.orc_nadd_out.argtypes = [C.c_void_p]
    lib.orc_nadd_out.restype = C.c_double
    lib.orc_set_substep_hook.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    _LIBS[key] = lib
    return lib


_HOOK = C.CFUNCTYPE(None, C.c_void_p, C.c_int)


class Oracle:
    """One CaMa-Flood model instance initialised exactly like CMF_DRV_INIT."""

    def __init__(self, casedir: str, nml: str = "input_cmf.nam", omp: bool = False):
        self.lib = _lib(omp)
        err = C.create_string_buffer(256)
        self.h = self.lib.orc_create(casedir.encode(), nml.encode(), err, 256)
        if not self.h:
            raise RuntimeError("oracle init failed: " + err.value.decode())
        d = (C.c_int * 11)()
        self.lib.orc_dims(self.h, d)
        (self.nx, self.ny, self.nlfp, self.nseqmax, self.nseqall, self.nseqriv,
         self.npthout, self.npthlev, self.ndam, self.upnmax, _) = list(d)

    def threads(self) -> int:
        return int(self.lib.orc_threads())

    def put_runoff(self, runoff_m3s: np.ndarray) -> None:
        a = np.ascontiguousarray(runoff_m3s, dtype=np.float64)
        assert a.shape == (self.nseqmax,)
        self.lib.orc_put_runoff_vec(self.h, a.ctypes.data_as(C.POINTER(C.c_double)))

    def put_runoff_map(self, runoff_map: np.ndarray) -> None:
        a = np.ascontiguousarray(runoff_map, dtype=np.float64).ravel()
        assert a.size == self.nx * self.ny
        self.lib.orc_put_runoff_map(self.h, a.ctypes.data_as(C.POINTER(C.c_double)))

    def advance(self):
        nt = C.c_int(0)
        dt = C.c_double(0.0)
        rc = self.lib.orc_physics_advance(self.h, C.byref(nt), C.byref(dt))
        if rc:
            raise RuntimeError(f"oracle advance failed rc={rc}")
        return nt.value, dt.value

    def stage(self) -> float:
        """Stage scheme + this domain's CFL minimum (before CMF_MPI_ADPSTP)."""
        return float(self.lib.orc_stage(self.h))

    def substeps(self, dt_min: float):
        nt = C.c_int(0)
        dt = C.c_double(0.0)
        self.lib.orc_substeps(self.h, dt_min, C.byref(nt), C.byref(dt))
        return nt.value, dt.value

    def write_restart(self, path: str, dbl: bool = True, stoonly: bool = False) -> None:
        """WRTE_REST_BIN (src/cmf_ctrl_restart_mod.F90:389-482) to `path` (+ `path`.pth)."""
        if self.lib.orc_write_restart(self.h, path.encode(), int(dbl), int(stoonly)) != 0:
            raise OSError(f"oracle: cannot write restart {path}")

    def read_restart(self, path: str, dbl: bool = True, stoonly: bool = False) -> None:
        """CMF_RESTART_INIT / READ_REST_BIN (src/cmf_ctrl_restart_mod.F90:91-204)."""
        if self.lib.orc_read_restart(self.h, path.encode(), int(dbl), int(stoonly)) != 0:
            raise OSError(f"oracle: cannot read restart {path}")

    def physics_fldstg(self) -> None:
        self.lib.orc_physics_fldstg(self.h)

    def calc_outpre(self) -> None:
        """CMF_CALC_OUTPRE (src/cmf_opt_outflw_mod.F90:308-421)."""
        self.lib.orc_calc_outpre(self.h)

    def put_runoff_grid(self, grid, inpmat=None, clean: bool = False) -> None:
        """CMF_FORCING_PUT (src/cmf_ctrl_forcing_mod.F90:716-831) of one runoff field PBUFF(NXIN,NYIN)
        given as [NYIN, NXIN]: ROFF_INTERP with inpmat = (nxin, nyin, inpx, inpy, inpa) ([INPN][N]
        arrays), else CONV_RESOL.  clean applies CMF_FORCING_GET's NaN/negative cleaning first."""
        g = np.array(grid, dtype=np.float64, order="C").ravel()
        if clean:
            self.lib.orc_forcing_clean(g.ctypes.data_as(C.POINTER(C.c_double)), g.size)
        if inpmat is None:
            self.put_runoff_map(g)
            return
        nxin, nyin, ix, iy, a = inpmat
        ix = np.ascontiguousarray(ix, dtype=np.int32)
        iy = np.ascontiguousarray(iy, dtype=np.int32)
        a = np.ascontiguousarray(a, dtype=np.float64)
        inpn = ix.size // self.nseqall
        self.lib.orc_roff_interp(self.h, g.ctypes.data_as(C.POINTER(C.c_double)), nxin, nyin, inpn,
                                 ix.ctypes.data_as(C.POINTER(C.c_int)), iy.ctypes.data_as(C.POINTER(C.c_int)),
                                 a.ctypes.data_as(C.POINTER(C.c_double)))

    def update_boundary(self, sealev=None, meansl=None) -> None:
        """CMF_BOUNDARY_UPDATE (src/cmf_ctrl_boundary_mod.F90:267-304)."""
        keep = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (sealev, meansl)]
        ptr = [None if a is None else a.ctypes.data_as(C.POINTER(C.c_double)) for a in keep]
        self.lib.orc_update_boundary(self.h, ptr[0], ptr[1])

    def diag_output(self, op: str) -> None:
        """CMF_DIAG_RESET_OUTPUT / CMF_DIAG_AVEMAX_OUTPUT / CMF_DIAG_GETAVE_OUTPUT
        (src/cmf_calc_diag_mod.F90:222-356): op = "reset", "avemax" or "getave"."""
        self.lib.orc_diag_output(self.h, {"reset": 0, "avemax": 1, "getave": 2}[op])

    def on_substep(self, fn) -> None:
        """Calls fn(it) after each sub-step's stage update, before the sub-step averages read its
        fields (it = 1..NT); None removes the hook."""
        if fn is None:
            self._hook = None
            self.lib.orc_set_substep_hook(self.h, None, None)
            return
        self._hook = _HOOK(lambda ctx, it: fn(it))
        self.lib.orc_set_substep_hook(self.h, C.cast(self._hook, C.c_void_p), None)

    def nadd_out(self) -> float:
        return float(self.lib.orc_nadd_out(self.h))

    def budget(self) -> dict:
        b = (C.c_double * 15)()
        self.lib.orc_budget(self.h, b)
        k = ["stopre", "stonxt", "stonew", "rivinf", "rivout", "stopre2", "stonew2", "rivsto", "fldsto",
             "fldare", "levsto", "dam_miss", "dt", "dt_min", "nadd"]
        return dict(zip(k, list(b)))

    def d(self, name: str) -> np.ndarray:
        n = C.c_int(0)
        p = self.lib.orc_darray(self.h, name.encode(), C.byref(n))
        if n.value < 0:
            raise KeyError(name)
        if n.value == 0:
            return np.zeros(0)
        return np.ctypeslib.as_array(p, shape=(n.value,)).copy()

    def i(self, name: str) -> np.ndarray:
        n = C.c_int(0)
        p = self.lib.orc_iarray(self.h, name.encode(), C.byref(n))
        if n.value < 0:
            raise KeyError(name)
        if n.value == 0:
            return np.zeros(0, dtype=np.int32)
        return np.ctypeslib.as_array(p, shape=(n.value,)).copy()
