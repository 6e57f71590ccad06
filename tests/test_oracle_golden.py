"""Pins the oracle (oracle/sf_oracle.c + oracle/oracle.py) to the reference's own outputs.

The fixtures were produced by running the reference's kernels (host-compiled from its
sources) under its own Python orchestration (tests/golden/make_golden.py).  The oracle must
reproduce them bit for bit: both sides evaluate the same IEEE-754 expressions in the same
order, with floating-point contraction disabled.
"""
import numpy as np
import pytest

import oracle as orc
from golden_io import load, boundary_dict


def _grid_from(d, pre="in_grid_"):
    L, M, N = int(d["in_L"]), int(d["in_M"]), int(d["in_N"])
    g = lambda k: d[pre + k]
    return orc.Grid(L, M, N, g("h"), g("pm"), g("pn"), g("on_u"), g("om_v"), g("fomn"), g("sc_r"),
                    g("sc_w"), g("Cs_r"), g("Cs_w"), float(g("hc")), int(d["in_Vtransform"]))


@pytest.mark.parametrize("tag", ["square", "nonsquare", "vt1"])
def test_oracle_main3d_matches_reference(tag):
    d = load("main3d_%s.npz" % tag)
    grid = _grid_from(d)
    B = orc.Boundary(boundary_dict(d, "in_bnd_"))
    init = {n: d["in_" + n] for n in ("zeta", "ubar", "vbar", "rzeta", "rubar", "rvbar", "u", "v",
                                      "ru", "rv", "W", "Huon", "Hvom", "Zt_avg1", "DU_avg1",
                                      "DV_avg1", "AKv")}
    O = orc.Ocean(grid, init)
    ct = orc.CompTimes(float(d["in_dt"]), int(d["in_ndtfast"]), int(d["in_nfast"]), d["in_w1"], d["in_w2"])
    orc.main3d(grid, B, O, ct, int(d["in_nsteps"]))
    for n in ("zeta", "ubar", "vbar", "rzeta", "rubar", "rvbar"):
        assert O.slots[n] == list(d["out_slots_" + n]), n
    for n in init:
        np.testing.assert_array_equal(getattr(O, n).reshape(-1), d["out_" + n].reshape(-1), err_msg=n)
    for n in ("z_w", "z_r", "Hz"):
        np.testing.assert_array_equal(getattr(grid, n).reshape(-1), d["out_" + n].reshape(-1), err_msg=n)
    assert ct.iic == int(d["out_iic"]) and ct.time == float(d["out_time"])
    assert ct.time2D == float(d["out_time2D"])


def test_reference_driver_matches_reference_main3d():
    """oracle/ref_driver.py (the reference's own kernels in main3d order, used as the timed CPU
    baseline) reproduces the reference's main3d run."""
    import ref_driver
    if not ref_driver.available():
        pytest.skip("oracle/_ref not built")
    d = load("main3d_square.npz")
    grid = _grid_from(d)
    B = orc.Boundary(boundary_dict(d, "in_bnd_"))
    names = ("zeta", "ubar", "vbar", "rzeta", "rubar", "rvbar", "u", "v", "ru", "rv", "W", "Huon",
             "Hvom", "Zt_avg1", "DU_avg1", "DV_avg1", "AKv")
    O = orc.Ocean(grid, {n: d["in_" + n] for n in names})
    ct = orc.CompTimes(float(d["in_dt"]), int(d["in_ndtfast"]), int(d["in_nfast"]), d["in_w1"], d["in_w2"])
    ref_driver.main3d(grid, B, O, ct, int(d["in_nsteps"]), omp=1)
    for n in names:
        np.testing.assert_array_equal(getattr(O, n).reshape(-1), d["out_" + n].reshape(-1), err_msg=n)
