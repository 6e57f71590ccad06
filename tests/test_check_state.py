"""Blow-up detection (sf_check_state): NaN, infinities and out-of-bound magnitudes in the
prognostic fields are reported as SF_ENONFINITE through the C ABI, naming the field and the
position of the first bad value.  Failures are made on the host (values planted in the inputs
before they are copied to the device, or the reference's own unstable step); no kernel is
made to fault."""
import numpy as np
import pytest


def _model(Lm=40, Mm=40, N=8, precision="fp32"):
    from sailfish_b200 import configs
    from sailfish_b200.model import Model
    cfg = configs.basin(Lm, Mm, N, 2.0e3, [(0.5, 0.5)], dt=120.0, ndtfast=10)
    m = Model(cfg["grid"], cfg["boundary"], cfg["dt"], cfg["ndtfast"], precision=precision)
    m.start()
    return m, cfg


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_clean_state_passes(precision):
    m, _ = _model(precision=precision)
    m.check_state()
    m.check_every = 1
    m.step(2)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("field,value", [("u", np.nan), ("v", np.inf), ("zeta", 1e4),
                                         ("ubar", -np.inf), ("u", 75.0)])
def test_planted_bad_value_is_reported(precision, field, value):
    from sailfish_b200._lib import SailfishError, SF_ENONFINITE
    m, cfg = _model(precision=precision)
    g = cfg["grid"]
    k, j, i = 3, 17, 23
    if field in ("u", "v"):
        host = np.zeros((g.N + 1, g.J, g.I))
        host[k, j, i] = value
        m.load({field: host})
        where = "level %d, j %d, i %d" % (k, j, i)
    else:
        host = np.zeros((3, g.J, g.I))
        host[m.slots[2], j, i] = value
        m.load({field: host})
        where = "level 0, j %d, i %d" % (j, i)
    with pytest.raises(SailfishError) as e:
        m.check_state()
    assert e.value.code == SF_ENONFINITE
    assert field in str(e.value) and where in str(e.value)


@pytest.mark.gpu
def test_first_bad_value_wins_and_the_flag_is_reset():
    from sailfish_b200._lib import SailfishError
    m, cfg = _model(precision="fp32")
    g = cfg["grid"]
    host = np.zeros((g.N + 1, g.J, g.I))
    host[5, 30, 2] = np.nan
    host[2, 10, 7] = np.nan            # the smaller flat index
    m.load({"u": host})
    with pytest.raises(SailfishError) as e:
        m.check_state()
    assert "level 2, j 10, i 7" in str(e.value)
    m.load({"u": np.zeros_like(host)})
    m.check_state()                    # a clean state after a failed check passes


@pytest.mark.gpu
def test_the_reference_blow_up_is_caught_during_the_step():
    """The reference's step semantics are unstable: a 1 cm surface bump on a 128 x 64 x 16
    basin goes out of bounds within a few steps.  With a check after every step the model
    stops at the first step whose state is out of bounds (found here by stepping a second
    model one step at a time and inspecting its fields on the host side) instead of running
    on."""
    import torch
    from sailfish_b200 import configs
    from sailfish_b200._lib import SailfishError, SF_ENONFINITE
    from sailfish_b200.model import Model
    cfg = configs.basin(128, 64, 16, 2.0e3, [(0.5, 0.5)], dt=240.0, ndtfast=30)
    g = cfg["grid"]
    bump = 1e-2 * np.exp(-((g.x - g.x.max() / 2) ** 2 + (g.y - g.y.max() / 2) ** 2) / (5e4) ** 2)

    def make():
        m = Model(g, cfg["boundary"], cfg["dt"], cfg["ndtfast"], precision="fp64")
        m.Zt_avg1.copy_(torch.from_numpy(bump.ravel()))
        return m

    def bad(m):
        sl = lambda n: getattr(m, n)[m.slots[2]]
        for t, b in ((sl("zeta"), m.surface_bound), (sl("ubar"), m.velocity_bound),
                     (sl("vbar"), m.velocity_bound), (m.u, m.velocity_bound),
                     (m.v, m.velocity_bound)):
            if not bool((t.abs() <= b).all()):
                return True
        return False

    ref = make()
    first = None
    for k in range(1, 9):
        ref.step(1)
        torch.cuda.synchronize()
        if bad(ref):
            first = k
            break
    assert first is not None, "the reference's step stayed bounded for 8 steps"
    m = make()
    m.check_every = 1
    with pytest.raises(SailfishError) as e:
        m.step(8)
    assert e.value.code == SF_ENONFINITE
    assert m.iic == first


@pytest.mark.gpu
def test_bad_bounds_are_rejected():
    import ctypes
    from sailfish_b200._lib import lib, SF_EINVAL
    m, _ = _model()
    st = ctypes.c_void_p(0)
    assert lib.sf_check_state(m.ctx.ptr, None, None, None, None, None, 0.0, 1.0, st) == SF_EINVAL
    assert lib.sf_check_state(m.ctx.ptr, None, None, None, None, None, 1.0, float("nan"),
                              st) == SF_EINVAL
