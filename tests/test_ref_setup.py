"""The oracle's restatement of the reference's host set-up (oracle/ref_setup.py), which the
benchmark's reference arm uses instead of the package, against the reference's own outputs
(tests/golden/setup.npz) and against the package's basins (same workload on both arms)."""
import numpy as np
import pytest

import ref_setup
from golden_io import load, BND_KEYS

S = load("setup.npz")
DEFAULT = {"isFsur": "Clo Clo Clo Clo", "isUbar": "Cla Clo Clo Clo", "isVbar": "Clo Clo Clo Clo",
           "isUvel": "Cla Clo Clo Clo", "isVvel": "Cla Clo Clo Clo"}   # utility/test.in:185-189


@pytest.mark.parametrize("nd", [10, 20, 30, 40, 60])
def test_weights_bit_exact(nd):
    nfast, w1, w2 = ref_setup.weights(nd)
    assert nfast == int(S["weights_%d_nfast" % nd])
    np.testing.assert_array_equal(w1, S["weights_%d_w1" % nd])
    np.testing.assert_array_equal(w2, S["weights_%d_w2" % nd])


@pytest.mark.parametrize("ts,tb", [(5.0, 0.4), (0.0, 0.0), (7.0, 2.0)])
def test_scoord_bit_exact(ts, tb):
    key = "coords_v4_%g_%g" % (ts, tb)
    for name, a in zip(("sc_r", "sc_w", "Cs_r", "Cs_w"), ref_setup.scoord(7, ts, tb)):
        np.testing.assert_array_equal(a, S[key + "_" + name], err_msg=name)


@pytest.mark.parametrize("Lm,Mm", [(12, 12), (16, 10), (9, 14)])
def test_lbc_lists_bit_exact(Lm, Mm):
    out = ref_setup.lbc_lists(Lm + 1, Mm + 1, DEFAULT)
    pre = "bnd_%dx%d_" % (Lm, Mm)
    for name in ("zetaBC", "ubarBC", "vbarBC", "uvelBC", "vvelBC"):
        for f in ("bcIdx", "bcIdx1", "bcIdx2", "bcIdxFieldIdx2", "bcIdxFieldType", "LBC"):
            np.testing.assert_array_equal(out["%s_%s" % (name, f)], S["%s%s_%s" % (pre, name, f)],
                                          err_msg="%s.%s" % (name, f))
    for f in BND_KEYS:
        np.testing.assert_array_equal(out[f], S[pre + f], err_msg=f)


def test_metrics_bit_exact():
    pre = "metrics_16x10_"
    on_u, om_v, fomn = ref_setup.metrics(S[pre + "pm"], S[pre + "pn"], S[pre + "f"])
    for k, a in (("on_u", on_u), ("om_v", om_v), ("fomn", fomn)):
        np.testing.assert_array_equal(a, S[pre + k], err_msg=k)


@pytest.mark.parametrize("name,shrink", [("basin4", 8), ("basin1", 4)])
def test_basin_matches_the_package_workload(name, shrink):
    """Both arms of the benchmark step the same basin: the oracle-side set-up gives the
    package's grid, tables, weights and boundary lists bit for bit."""
    from sailfish_b200 import configs, host
    Lm, Mm, N, dx, mounts, dt, nd = ref_setup.BASINS[name]
    cfg = configs.basin(Lm // shrink, Mm // shrink, N, dx, list(mounts), dt, nd)
    g, B = cfg["grid"], cfg["boundary"]
    b = ref_setup.basin(name, shrink)
    assert (b["L"], b["M"], b["N"], b["dt"], b["ndtfast"]) == (g.L, g.M, g.N, cfg["dt"],
                                                                 cfg["ndtfast"])
    for k in ("h", "pm", "pn", "on_u", "om_v", "fomn", "sc_r", "sc_w", "Cs_r", "Cs_w"):
        np.testing.assert_array_equal(np.asarray(b[k]).ravel(), np.asarray(getattr(g, k)).ravel(),
                                      err_msg=k)
    assert b["hc"] == g.hc and b["Vtransform"] == g.Vtransform
    nf, w1, w2 = host.set_weights(nd)
    rf, r1, r2 = ref_setup.weights(nd)
    assert nf == rf and np.array_equal(w1, r1) and np.array_equal(w2, r2)
    for f in BND_KEYS:
        np.testing.assert_array_equal(b["lists"][f], getattr(B, f), err_msg=f)
    for name_ in ("zetaBC", "uvelBC", "vvelBC"):
        for f in ("bcIdxFieldIdx2", "bcIdxFieldType"):
            np.testing.assert_array_equal(b["lists"]["%s_%s" % (name_, f)],
                                          getattr(getattr(B, name_), f), err_msg=name_ + f)
