"""Writes the golden fixture: a tiny seeded case in the reference's file formats (mini_case/) and the
oracle's outputs over 12 hourly coupling steps (golden_mini.npz).

    python tests/golden/make_golden.py

The reference (Fortran) cannot be built on this machine, so these vectors come from the oracle,
the CPU restatement in oracle/; they pin the oracle and the GPU path against regressions and
against each other, not against a run of the Fortran reference (parity unpinned).
"""
from __future__ import annotations

import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "cama-flood_v4_b200"), os.path.join(ROOT, "oracle")]

NSTEPS = 12


def spec():
    from cmf_b200 import synth

    s = synth.spec_config1(seed=11, scale=0.03)     # 43x22 grid, levees, dams, bifurcation
    s.name = "golden_mini"
    s.rivhgt_scale = 0.3                             # floodplain flow within the first hours
    return s


def main():
    from cmf_b200 import synth
    from oracle import Oracle

    case = os.path.join(HERE, "mini_case")
    if os.path.exists(case):
        shutil.rmtree(case)
    synth.write_case(synth.make_case(spec()), case)
    o = Oracle(case)
    gr = o.d("grarea")
    gen = synth.AR1GammaRunoff(o.nseqall, 5)
    runoff = np.stack([np.maximum((gen.next().astype(np.float64) * 8.0 * gr) / 86400000.0, 0.0) for _ in range(NSTEPS)])
    nt, dt = [], []
    for k in range(NSTEPS):
        o.put_runoff(runoff[k])
        a, b = o.advance()
        nt.append(a)
        dt.append(b)
    out = {"runoff": runoff, "nt": np.array(nt), "dt": np.array(dt)}
    for f in ("rivsto", "fldsto", "rivout", "fldout", "rivdph", "flddph", "levsto", "damsto", "pthflw",
              "rivout_aavg", "storge_amax"):
        out[f] = o.d(f)
    np.savez_compressed(os.path.join(HERE, "golden_mini.npz"), **out)
    print("cells", o.nseqall, "paths", o.npthout, "dams", o.ndam, "NT", nt)


if __name__ == "__main__":
    main()
