"""Ensembles (config 2): members of different sizes and N stepped together through the
pooled, block-mapped kernels give exactly what each member gives stepped alone (FP64:
bit-exact; the single-grid FP64 path is itself bit-exact to the reference)."""
import numpy as np
import pytest

from sailfish_b200 import configs


def small_members():
    out = []
    for Lm, Mm, N in ((20, 20, 6), (33, 17, 8), (12, 25, 5)):
        cfg = configs.basin(Lm, Mm, N, 2.0e4, [(0.5, 0.5)], dt=240.0, ndtfast=10)
        g = cfg["grid"]
        z0 = 1e-3 * np.exp(-((g.x - g.x.mean()) ** 2 + (g.y - g.y.mean()) ** 2) / (1e5) ** 2)
        out.append((g, cfg["boundary"], z0))
    return out


def test_member_recipe_is_seeded():
    from sailfish_b200 import ensemble
    a = ensemble.ensemble_members(seed=5, n=4)
    b = ensemble.ensemble_members(seed=5, n=4)
    for (g1, _, z1), (g2, _, z2) in zip(a, b):
        assert (g1.L, g1.M, g1.N) == (g2.L, g2.M, g2.N)
        np.testing.assert_array_equal(z1, z2)
    assert all(64 <= g.L - 1 <= 512 and 32 <= g.M - 1 <= 256 and g.N in (16, 32) for g, _, _ in a)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_ensemble_matches_members_stepped_alone(precision):
    import torch
    from sailfish_b200 import ensemble
    from sailfish_b200.model import Model
    members = small_members()
    ens = ensemble.make(members, precision=precision, dt=240.0, ndtfast=10)
    ens.step(3)
    torch.cuda.synchronize()
    for m, (g, b, z0) in enumerate(members):
        single = Model(g, b, 240.0, 10, precision=precision)
        zt = torch.from_numpy(np.ascontiguousarray(z0, np.float64).ravel()).cuda()
        single.Zt_avg1.copy_(zt)
        for k in range(3):
            single.zeta[k].view(-1).copy_(zt.to(single.tdtype))
        single.step(3)
        torch.cuda.synchronize()
        for name in ("zeta", "ubar", "vbar", "u", "v", "W", "Zt_avg1", "DU_avg1", "z_w", "Hz"):
            if name in Model.NAMES2:
                a = ens.member(name, m, 2)
                bb = single._slot(name, 2)
            else:
                a = ens.member(name, m)
                bb = getattr(single, name).view(a.shape)
            a, bb = a.double().cpu().numpy(), bb.double().cpu().numpy().reshape(a.shape)
            if precision == "fp64":
                np.testing.assert_array_equal(a, bb, err_msg="member %d %s" % (m, name))
            else:
                # the reference's step goes non-finite on non-square grids: same places both ways
                np.testing.assert_array_equal(np.isfinite(a), np.isfinite(bb))
                fin = np.isfinite(bb)
                scale = max(np.abs(bb[fin]).max(initial=0.0), 1e-30)
                np.testing.assert_allclose(a[fin], bb[fin], rtol=0, atol=1e-5 * scale,
                                           err_msg="member %d %s" % (m, name))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_rhs3d_tile_variants_agree_and_autotune_picks_one(precision):
    import torch
    from sailfish_b200 import autotune, ensemble
    from sailfish_b200._lib import lib
    members = small_members()
    ens = ensemble.make(members, precision=precision, dt=240.0, ndtfast=10)
    ens.step(2)
    out = {}
    for v in (0, 1, 2, 3):
        assert lib.sf_ctx_set_tile(ens.ctx.ptr, v) == 0
        ens.ru.zero_()
        ens.rv.zero_()
        autotune._time(lambda: lib.sf_rhs3d(ens.ctx.ptr, ens._p(ens.u), ens._p(ens.v),
                                            ens._p(ens.Huon), ens._p(ens.Hvom), ens._p(ens.W),
                                            ens._p(ens.Hz), ens._p(ens.ru), ens._p(ens.rv),
                                            ctypes_stream()), 1)
        out[v] = (ens.ru.clone(), ens.rv.clone())
    # (the non-square member's state is not finite after two steps of the reference's scheme:
    # NaNs must sit in the same places)
    for v in (1, 2, 3):
        tol = dict(rtol=0, atol=0) if precision == "fp64" else dict(rtol=1e-5, atol=1e-6)
        for k in range(2):
            torch.testing.assert_close(out[v][k], out[0][k], equal_nan=True, **tol)
    times = autotune.tune_rhs3d(ens, reps=2)
    assert set(times) == {0, 1, 2, 3} and ens.rhs_tile in times


def ctypes_stream():
    import ctypes
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_roms_ensemble_matches_members_stepped_alone(precision):
    """The ROMS-form step on an ensemble (pooled, block-mapped kernels) against each member
    stepped alone in the ROMS form with the same wind and drag: bit for bit in FP64; in FP32
    the pooled and single-grid kernels may contract different products into FMAs."""
    import torch
    from sailfish_b200 import ensemble
    from sailfish_b200.model import Model
    members = small_members()
    ens = ensemble.make(members, precision=precision, dt=240.0, ndtfast=10, semantics="roms")
    ensemble.roms_forcing(ens, tau0=0.1, rdrag2=3e-3)
    ens.step(4)
    torch.cuda.synchronize()
    c = ens.ctx
    su = ens.sustr.double().cpu().numpy()
    for m, (g, b, z0) in enumerate(members):
        single = Model(g, b, 240.0, 10, precision=precision, semantics="roms")
        single.set_forcing(su[c.off2[m]:c.off2[m] + g.s2], np.zeros(g.s2), 3e-3)
        zt = torch.from_numpy(np.ascontiguousarray(z0, np.float64).ravel()).cuda()
        single.Zt_avg1.copy_(zt)
        for k in range(3):
            single.zeta[k].view(-1).copy_(zt.to(single.tdtype))
        single.step(4)
        torch.cuda.synchronize()
        for name in ("zeta", "ubar", "vbar", "u", "v", "W", "Zt_avg1", "DU_avg1", "z_w", "Hz"):
            if name in Model.NAMES2:
                a = ens.member(name, m, 1)
                bb = single._slot(name, 1)
            else:
                a = ens.member(name, m)
                bb = getattr(single, name).view(a.shape)
            a, bb = a.double().cpu().numpy(), bb.double().cpu().numpy().reshape(a.shape)
            assert np.isfinite(bb).all(), "member %d %s" % (m, name)
            if precision == "fp64":
                np.testing.assert_array_equal(a, bb, err_msg="member %d %s" % (m, name))
            else:
                scale = max(np.abs(bb).max(), 1e-30)
                np.testing.assert_allclose(a, bb, rtol=0, atol=1e-5 * scale,
                                           err_msg="member %d %s" % (m, name))
        u = ens.member("u", m).double().cpu().numpy()
        assert np.abs(u).max() > 0      # the wind has moved every member

