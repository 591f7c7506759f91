"""ctypes mirror of include/cmf_gpu.h (the C ABI of the B200 physics time step).

The structs below must match the header field for field; tests/test_abi.py checks the symbol list
and the struct sizes against the header.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libcmf_b200.so")

i32p = C.POINTER(C.c_int32)
f64p = C.POINTER(C.c_double)


class Dims(C.Structure):
    _fields_ = [(n, C.c_int32) for n in (
        "nseqall", "nseqriv", "nseqmax", "nlfp", "upnmax", "npthout", "npthlev", "onmax", "inmax", "ndam", "nmembers")]


class Params(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("pgrv", "pmanfld", "pdstmth", "pcadp", "pminslp", "dfrcinc")]


class Opts(C.Structure):
    _fields_ = [(n, C.c_int32) for n in (
        "ladpstp", "lfldout", "lpthout", "ldamout", "llevee", "lspamat",
        "lkine", "lslpmix", "lstg_es", "lgdwdly", "lrosplit", "lwevap", "lupsinf", "lheatlink", "ltrace", "lslopemouth",
        "ldamh22", "ldamyby", "ldiag", "launch_mode", "device", "block_size", "ldiag_output")]


MAP_FIELDS = [
    ("i1next", i32p), ("i1upst", i32p), ("i1upn", i32p), ("i2mask", i32p),
    ("rivelv", f64p), ("elevtn", f64p), ("nxtdst", f64p), ("rivwth", f64p), ("rivhgt", f64p), ("rivlen", f64p),
    ("rivman", f64p), ("grarea", f64p), ("rivstomax", f64p), ("dwnelv", f64p),
    ("fldstomax", f64p), ("fldgrd", f64p), ("fldhgt", f64p),
    ("pth_upst", i32p), ("pth_down", i32p), ("pth_dst", f64p), ("pth_elv", f64p), ("pth_wth", f64p), ("pth_man", f64p),
    ("i1p_out", i32p), ("i1p_outn", i32p), ("i1p_inf", i32p), ("i1p_infn", i32p),
    ("levhgt", f64p), ("levfrc", f64p), ("bashgt", f64p), ("levdst", f64p), ("levbassto", f64p), ("levtopsto", f64p),
    ("levfilsto", f64p),
    ("damseq", i32p), ("damstat", i32p), ("i1dam", i32p),
    ("dam_qn", f64p), ("dam_qf", f64p), ("dam_qa", f64p), ("dam_convol", f64p), ("dam_fldvol", f64p),
    ("dam_emevol", f64p), ("dam_norvol", f64p), ("dam_adjvol", f64p), ("dam_r_volupa", f64p),
]


class MapPtrs(C.Structure):
    _fields_ = MAP_FIELDS


STATE_FIELDS = ["rivsto", "fldsto", "rivout", "fldout", "rivout_pre", "fldout_pre", "rivdph_pre", "fldsto_pre",
                "pthflw", "pthflw_pre", "damsto", "daminf", "levsto"]


class StatePtrs(C.Structure):
    _fields_ = [(n, f64p) for n in STATE_FIELDS]


DIAG_FIELDS = ["rivdph", "flddph", "fldfrc", "fldare", "sfcelv", "storge", "rivvel",
               "rivinf", "fldinf", "pthout", "outflw", "pthflwsum", "levdph",
               "rivout_aavg", "fldout_aavg", "outflw_aavg", "rivvel_aavg", "pthout_aavg",
               "gdwrtn_aavg", "runoff_aavg", "rofsub_aavg", "daminf_aavg",
               "storge_amax", "outflw_amax", "rivdph_amax", "pthflw_aavg", "pthflwsum_aavg"]


class DiagPtrs(C.Structure):
    _fields_ = [(n, f64p) for n in DIAG_FIELDS]


DIAG_OUT_FIELDS = ["rivout_oavg", "fldout_oavg", "outflw_oavg", "rivvel_oavg", "pthout_oavg",
                   "gdwrtn_oavg", "runoff_oavg", "rofsub_oavg", "daminf_oavg",
                   "storge_omax", "outflw_omax", "rivdph_omax", "pthflw_oavg", "nadd_out"]


class DiagOutPtrs(C.Structure):
    _fields_ = [(n, f64p) for n in DIAG_OUT_FIELDS]


BUDGET_FIELDS = ["stopre", "stonxt", "stonew", "rivinf", "rivout", "stopre2", "stonew2", "rivsto", "fldsto",
                 "fldare", "levsto", "dam_miss"]


class Budget(C.Structure):
    _fields_ = [(n, C.c_double) for n in BUDGET_FIELDS]


class Schedule(C.Structure):
    _fields_ = [("mode", C.c_int32), ("flux_block", C.c_int32), ("rate_block", C.c_int32), ("store_block", C.c_int32),
                ("profile", C.c_int32), ("tuned", C.c_int32), ("candidates", C.c_int32),
                ("best_us_per_substep", C.c_double), ("worst_us_per_substep", C.c_double)]


class StageDevArgs(C.Structure):
    _fields_ = [("nseqall", C.c_int32), ("nseqriv", C.c_int32), ("nlfp", C.c_int32), ("ladpstp", C.c_int32),
                ("dt_def", C.c_double), ("pgrv", C.c_double), ("pdstmth", C.c_double), ("pcadp", C.c_double),
                ("dfrcinc", C.c_double)] + [(n, C.c_void_p) for n in (
        "rivstomax", "rivlen", "rivwth", "grarea", "rivelv", "nxtdst", "fldstomax", "fldgrd", "i2mask",
        "rivsto", "fldsto", "rivdph", "flddph", "fldfrc", "fldare", "sfcelv", "storge", "dt_min_out", "stream")]


EXPORTS = [
    "cmf_gpu_create", "cmf_gpu_destroy", "cmf_gpu_ctx_set_state", "cmf_gpu_ctx_get_state", "cmf_gpu_ctx_put_runoff",
    "cmf_gpu_ctx_physics_advance", "cmf_gpu_ctx_get_diag", "cmf_gpu_ctx_advance_device", "cmf_gpu_ctx_synchronize",
    "cmf_gpu_ctx_last_nt", "cmf_gpu_ctx_stream", "cmf_gpu_ctx_kernel_launches", "cmf_gpu_ctx_block_size",
    "cmf_gpu_ctx_stage", "cmf_gpu_ctx_substeps", "cmf_gpu_ctx_counters", "cmf_gpu_ctx_time_phases",
    "cmf_gpu_init", "cmf_gpu_set_state", "cmf_gpu_get_state", "cmf_gpu_put_runoff", "cmf_gpu_physics_advance",
    "cmf_gpu_get_diag", "cmf_gpu_finalize", "cmf_gpu_strerror", "cmf_gpu_last_error", "cmf_gpu_abi_version",
    "cmf_host_load", "cmf_host_free", "cmf_host_describe", "cmf_host_state", "cmf_host_conv_resol", "cmf_host_grid",
    "cmf_gpu_stage_noalloc", "cmf_gpu_ctx_nt_stats", "cmf_gpu_ctx_diag_output", "cmf_gpu_ctx_get_diag_output",
    "cmf_gpu_diag_output", "cmf_gpu_get_diag_output", "cmf_gpu_ctx_persist_selftest", "cmf_gpu_ctx_launch_mode",
    "cmf_gpu_ctx_get_schedule", "cmf_gpu_ctx_set_schedule", "cmf_gpu_ctx_put_runoff_async",
    "cmf_gpu_ctx_advance_async", "cmf_gpu_ctx_wait", "cmf_gpu_ctx_get_diag_async", "cmf_gpu_ctx_io_wait",
]

_lib = None


def load(build_if_missing: bool = True):
    """Loads the in-tree library.  Raises if it is missing: there is no fallback path."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        if not build_if_missing:
            raise RuntimeError(f"{LIB_PATH} is not built")
        import importlib.util

        spec = importlib.util.spec_from_file_location("cmf_build", os.path.join(os.path.dirname(_HERE), "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    lib = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    lib.cmf_gpu_create.argtypes = [C.POINTER(Dims), C.POINTER(Params), C.POINTER(MapPtrs), C.POINTER(Opts), C.POINTER(vp)]
    lib.cmf_gpu_destroy.argtypes = [vp]
    lib.cmf_gpu_ctx_set_state.argtypes = [vp, C.POINTER(StatePtrs)]
    lib.cmf_gpu_ctx_get_state.argtypes = [vp, C.POINTER(StatePtrs)]
    lib.cmf_gpu_ctx_put_runoff.argtypes = [vp, f64p, f64p]
    lib.cmf_gpu_ctx_physics_advance.argtypes = [vp, C.c_double, i32p, f64p, C.POINTER(Budget)]
    lib.cmf_gpu_ctx_get_diag.argtypes = [vp, C.POINTER(DiagPtrs)]
    lib.cmf_gpu_ctx_put_runoff_async.argtypes = [vp, f64p]
    lib.cmf_gpu_ctx_advance_async.argtypes = [vp, C.c_double]
    lib.cmf_gpu_ctx_wait.argtypes = [vp, i32p, f64p, C.POINTER(Budget)]
    lib.cmf_gpu_ctx_get_diag_async.argtypes = [vp, C.POINTER(DiagPtrs)]
    lib.cmf_gpu_ctx_io_wait.argtypes = [vp]
    lib.cmf_gpu_ctx_advance_device.argtypes = [vp, C.c_double, C.c_int32, vp, C.c_int64]
    lib.cmf_gpu_ctx_synchronize.argtypes = [vp]
    lib.cmf_gpu_ctx_last_nt.argtypes = [vp, i32p, f64p]
    lib.cmf_gpu_ctx_stream.argtypes = [vp]
    lib.cmf_gpu_ctx_stream.restype = vp
    lib.cmf_gpu_ctx_kernel_launches.argtypes = [vp]
    lib.cmf_gpu_ctx_kernel_launches.restype = C.c_int64
    lib.cmf_gpu_ctx_block_size.argtypes = [vp]
    lib.cmf_gpu_ctx_stage.argtypes = [vp, C.c_double, f64p]
    lib.cmf_gpu_ctx_substeps.argtypes = [vp, C.c_double, C.c_double, i32p, f64p, C.POINTER(Budget)]
    lib.cmf_gpu_ctx_counters.argtypes = [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    lib.cmf_gpu_ctx_time_phases.argtypes = [vp, C.c_double, C.c_int32, f64p]
    lib.cmf_gpu_ctx_nt_stats.argtypes = [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.c_int32]
    lib.cmf_gpu_ctx_persist_selftest.argtypes = [vp, C.c_int64]
    lib.cmf_gpu_ctx_get_schedule.argtypes = [vp, C.POINTER(Schedule)]
    lib.cmf_gpu_ctx_set_schedule.argtypes = [vp, C.POINTER(Schedule)]
    lib.cmf_gpu_schedule_cache_clear.restype = None
    lib.cmf_gpu_ctx_launch_mode.argtypes = [vp]
    lib.cmf_gpu_ctx_diag_output.argtypes = [vp, C.c_int32]
    lib.cmf_gpu_ctx_get_diag_output.argtypes = [vp, C.POINTER(DiagOutPtrs)]
    lib.cmf_gpu_diag_output.argtypes = [C.c_int32]
    lib.cmf_gpu_get_diag_output.argtypes = [C.POINTER(DiagOutPtrs)]
    lib.cmf_gpu_batch_create.argtypes = [C.POINTER(vp), C.c_int32, C.POINTER(vp)]
    lib.cmf_gpu_batch_launch.argtypes = [vp, C.c_double]
    lib.cmf_gpu_batch_advance.argtypes = [vp, C.c_double, i32p, f64p, C.POINTER(Budget)]
    lib.cmf_gpu_batch_synchronize.argtypes = [vp]
    lib.cmf_gpu_batch_stream.argtypes = [vp]
    lib.cmf_gpu_batch_stream.restype = vp
    lib.cmf_gpu_batch_destroy.argtypes = [vp]
    lib.cmf_gpu_batch_destroy.restype = None
    lib.cmf_gpu_init.argtypes = [C.POINTER(Dims), C.POINTER(Params), C.POINTER(MapPtrs), C.POINTER(Opts)]
    lib.cmf_gpu_set_state.argtypes = [C.POINTER(StatePtrs)]
    lib.cmf_gpu_get_state.argtypes = [C.POINTER(StatePtrs)]
    lib.cmf_gpu_put_runoff.argtypes = [f64p, f64p]
    lib.cmf_gpu_physics_advance.argtypes = [C.c_double, i32p, f64p, C.POINTER(Budget)]
    lib.cmf_gpu_get_diag.argtypes = [C.POINTER(DiagPtrs)]
    lib.cmf_gpu_stage_noalloc.argtypes = [C.POINTER(StageDevArgs)]
    lib.cmf_gpu_strerror.argtypes = [C.c_int]
    lib.cmf_gpu_strerror.restype = C.c_char_p
    lib.cmf_gpu_last_error.restype = C.c_char_p
    lib.cmf_host_load.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(vp)]
    lib.cmf_host_free.argtypes = [vp]
    lib.cmf_host_describe.argtypes = [vp, C.POINTER(Dims), C.POINTER(Params), C.POINTER(MapPtrs), C.POINTER(Opts), f64p]
    lib.cmf_host_state.argtypes = [vp, C.POINTER(StatePtrs)]
    lib.cmf_host_conv_resol.argtypes = [vp, f64p, f64p]
    lib.cmf_host_grid.argtypes = [vp, i32p, i32p, i32p, i32p]
    lib.cmf_host_write_restart.argtypes = [vp, C.POINTER(StatePtrs), C.c_char_p, C.c_int32, C.c_int32]
    lib.cmf_host_read_restart.argtypes = [vp, C.POINTER(StatePtrs), C.c_char_p, C.c_int32, C.c_int32]
    lib.cmf_host_map_to_vec.argtypes = [vp, C.POINTER(C.c_float), f64p]
    lib.cmf_gpu_ctx_calc_outpre.argtypes = [vp]
    lib.cmf_gpu_ctx_set_runoff_map.argtypes = [vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, i32p, i32p, f64p, C.c_double]
    lib.cmf_gpu_ctx_put_runoff_grid.argtypes = [vp, vp, C.c_int32, C.c_int32, C.c_int32]
    lib.cmf_host_read_inpmat.argtypes = [vp, C.c_char_p, C.c_int32, i32p, i32p, f64p]
    lib.cmf_host_drofunit.argtypes = [vp]
    lib.cmf_host_drofunit.restype = C.c_double
    lib.cmf_gpu_ctx_update_boundary.argtypes = [vp, f64p, f64p]
    _lib = lib
    return lib


def check(rc: int, what: str = "") -> None:
    if rc != 0:
        lib = load()
        raise RuntimeError(f"{what}: status {rc} ({lib.cmf_gpu_strerror(rc).decode()}): {lib.cmf_gpu_last_error().decode()}")
