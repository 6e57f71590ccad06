"""Host set-up routines against the reference's own outputs (tests/golden/setup.npz)."""
import numpy as np
import pytest

from golden_io import load
from sailfish_b200 import host

S = load("setup.npz")


@pytest.mark.parametrize("nd", [10, 20, 30, 40, 60])
def test_set_weights_bit_exact(nd):
    nfast, w1, w2 = host.set_weights(nd)
    assert nfast == int(S["weights_%d_nfast" % nd])
    np.testing.assert_array_equal(w1, S["weights_%d_w1" % nd])
    np.testing.assert_array_equal(w2, S["weights_%d_w2" % nd])


@pytest.mark.parametrize("vs,ts,tb", [(1, 5.0, 0.4), (1, 0.0, 0.0), (2, 5.0, 0.4), (2, 3.0, 0.0),
                                      (3, 0.65, 0.58), (4, 5.0, 0.4), (4, 0.0, 0.0), (4, 7.0, 2.0)])
def test_set_coords_bit_exact(vs, ts, tb):
    out = host.set_coords(7, vs, ts, tb)
    key = "coords_v%d_%g_%g" % (vs, ts, tb)
    for name, a in zip(("sc_r", "sc_w", "Cs_r", "Cs_w"), out):
        np.testing.assert_array_equal(a, S[key + "_" + name], err_msg=name)


@pytest.mark.parametrize("Lm,Mm", [(12, 12), (16, 10), (9, 14)])
def test_boundary_bit_exact(Lm, Mm):
    B = host.Boundary(Lm + 1, Mm + 1)
    pre = "bnd_%dx%d_" % (Lm, Mm)
    for name in ("zetaBC", "ubarBC", "vbarBC", "uvelBC", "vvelBC"):
        bc = getattr(B, name)
        for f in ("bcIdx", "bcIdx1", "bcIdx2", "bcIdxFieldIdx2", "bcIdxFieldType", "LBC"):
            np.testing.assert_array_equal(getattr(bc, f), S["%s%s_%s" % (pre, name, f)],
                                          err_msg="%s.%s" % (name, f))
    for f in ("zetaClosedOrGradientBCIdx1", "zetaClosedOrGradientBCIdx2", "zetaClampedBCIdx1",
              "ubarClosedBCIdx1", "vbarClosedBCIdx1", "ubarClampedBCIdx1", "vbarClampedBCIdx1",
              "ubarGradientBCIdx1", "ubarGradientBCIdx2", "vbarGradientBCIdx1", "vbarGradientBCIdx2"):
        np.testing.assert_array_equal(getattr(B, f), S[pre + f], err_msg=f)


def test_metrics_bit_exact():
    pre = "metrics_16x10_"
    m = host.update_metrics(S[pre + "pm"], S[pre + "pn"], S[pre + "f"])
    for k in ("on_u", "om_v", "fomn", "om_u", "on_v", "omn"):
        np.testing.assert_array_equal(m[k], S[pre + k], err_msg=k)


def test_decode_lbc_rejects_unknown():
    with pytest.raises(ValueError):
        host.decode_lbc("XYZ")
    assert host.decode_lbc("cla") == host.bcClamped + host.bcAcquire
