"""The C-ABI library loads without a GPU and exports every entry point include/cmf_gpu.h declares;
the ctypes mirror matches the header's structs."""
from __future__ import annotations

import ctypes as C
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    txt = open(os.path.join(ROOT, "include", "cmf_gpu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = set(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\**\s*(cmf_[a-z0-9_]+)\s*\(", txt, flags=re.M))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    from cmf_b200 import _abi

    lib = _abi.load()
    declared = _declared_functions()
    assert len(declared) >= 30
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_abi.EXPORTS) <= set(declared)


def _struct_fields(name):
    txt = open(os.path.join(ROOT, "include", "cmf_gpu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    body = re.search(r"typedef struct " + name + r" \{(.*?)\} " + name + ";", txt, flags=re.S).group(1)
    fields = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        decl = re.sub(r"\b(const|int32_t|int64_t|double)\b", "", decl)
        fields += [f.strip().lstrip("*").strip() for f in decl.split(",")]
    return fields


def test_ctypes_structs_match_header():
    from cmf_b200 import _abi

    for cname, py in [("cmf_dims", _abi.Dims), ("cmf_params", _abi.Params), ("cmf_opts", _abi.Opts),
                      ("cmf_map_ptrs", _abi.MapPtrs), ("cmf_state_ptrs", _abi.StatePtrs),
                      ("cmf_diag_ptrs", _abi.DiagPtrs), ("cmf_budget", _abi.Budget),
                      ("cmf_diag_out_ptrs", _abi.DiagOutPtrs), ("cmf_schedule", _abi.Schedule)]:
        assert _struct_fields(cname) == [f[0] for f in py._fields_], cname


def test_abi_version_and_errors_without_device():
    from cmf_b200 import _abi

    lib = _abi.load()
    assert lib.cmf_gpu_abi_version() == 2
    assert lib.cmf_gpu_strerror(-2) == b"option combination not supported by the GPU path"
    assert lib.cmf_gpu_set_state(None) == -3        # no default context yet: CMF_E_STATE


def test_unsupported_options_are_refused(case_dirs):
    """cmf_gpu_create validates options before touching a device (negative status, no fallback)."""
    from cmf_b200 import HostModel, _abi

    h = HostModel(case_dirs["cfg0"])
    lib = _abi.load()
    opts = _abi.Opts.from_buffer_copy(h.opts)
    opts.lkine = 1
    ctx = C.c_void_p()
    rc = lib.cmf_gpu_create(C.byref(h.dims), C.byref(h.params), C.byref(h.maps), C.byref(opts), C.byref(ctx))
    assert rc == -2 and not ctx.value
    assert b"LKINE" in lib.cmf_gpu_last_error()
