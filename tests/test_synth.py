"""The synthetic-case generator's native loops (forest growth, upstream-area accumulation,
elevation walk) against their Python statements, and the committed golden case regenerated
byte for byte."""
from __future__ import annotations

import filecmp
import os

import numpy as np
import pytest

from cmf_b200 import synth

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("mk", [lambda: synth.spec_config0(seed=0), lambda: synth.spec_config1(seed=1, scale=0.1),
                                lambda: synth.spec_config4(seed=4, scale=0.04)])
def test_native_loops_equal_python(mk):
    spec = mk()
    rng = np.random.default_rng(spec.seed)
    land = synth._land_mask(spec, rng)
    mouths = synth._mouths(spec, land, rng)
    state = rng.bit_generator.state
    down, order = synth._grow_forest(land, mouths, rng)
    rng.bit_generator.state = state
    down_py, order_py = synth._grow_forest_py(land, mouths, rng)
    assert np.array_equal(down, down_py) and np.array_equal(order, order_py)
    assert order.size == int(np.sum(down > -2)) > 0
    n = down.size
    r2 = np.random.default_rng(5)
    upa = r2.lognormal(0.0, 0.2, n)
    slope, length = r2.uniform(1e-5, 1e-3, n), 15000.0 * r2.lognormal(0.0, 0.5, n)
    a, b = upa.copy(), upa.copy()
    synth._accumulate(order, down, a)
    synth._accumulate_py(order, down, b)
    assert np.array_equal(a.view(np.int64), b.view(np.int64))
    e1, e2 = np.zeros(n), np.zeros(n)
    synth._elevation(order, down, slope, length, e1)
    synth._elevation_py(order, down, slope, length, e2)
    assert np.array_equal(e1.view(np.int64), e2.view(np.int64))


def test_golden_case_regenerates_byte_for_byte(tmp_path):
    import sys

    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_golden

    out = str(tmp_path / "mini")
    synth.write_case(synth.make_case(make_golden.spec()), out)
    ref = os.path.join(HERE, "golden", "mini_case")
    names = sorted(os.listdir(ref))
    assert names == sorted(os.listdir(out))
    match, mismatch, errors = filecmp.cmpfiles(ref, out, names, shallow=False)
    assert not mismatch and not errors, (mismatch, errors)


def test_config4_spec_counts():
    s = synth.spec_config4()
    assert (s.nx, s.ny, s.npthout, s.ndam, s.npthlev) == (7200, 3600, 100_000, 10_000, 5)
    assert abs(s.land_frac * s.nx * s.ny - 6e6) < 1
    small = synth.spec_config4(scale=0.1)
    assert (small.nx, small.ny, small.npthout, small.ndam) == (720, 360, 1000, 100)
