"""The ROMS-form barotropic step (semantics "roms"): wind stress, quadratic bottom drag,
Coriolis and ROMS signs, restated from the reference's ROMS pseudo-code
(obsolete/step2d_LF_AM3.h.py, nonlinear/set_vbc.py) in oracle/roms_oracle.py.

CPU: the oracle conserves volume in a closed basin, and its stability limit is the one the
von Neumann analysis of the same scheme gives (an independent derivation of the time stepping).
GPU: the CUDA kernels against the oracle (FP64, bit for bit) and the FP32 form against FP64."""
import numpy as np
import pytest

import roms_oracle as ro


def _basin(Lm=40, Mm=30, dx=5e3, h=4000.0, f=True):
    from sailfish_b200 import configs
    cfg = configs.basin(Lm, Mm, 5, dx, [], dt=30.0, ndtfast=1, hflat=h)
    g = cfg["grid"]
    G = dict(h=g.h, pm=g.pm, pn=g.pn, on_u=g.on_u, om_v=g.om_v, fomn=g.fomn if f else 0 * g.fomn)
    return cfg, g, G


def _wind(g, tau0=0.1):
    Ly = (g.M - 1) * (1.0 / g.pn.flat[0])
    return tau0 * np.cos(np.pi * g.y / Ly) / 1025.0       # kinematic: tau / rho0


def test_oracle_conserves_volume_with_wind_drag_and_coriolis():
    cfg, g, G = _basin()
    S = ro.State(g.J, g.I)
    su = _wind(g)
    sv = 0.3 * su
    v0 = ro.volume(G, S.zeta[1])
    ro.main2d(G, S, 300, 15.0, su, sv, 3e-3)
    assert np.isfinite(S.zeta[1]).all() and np.abs(S.ubar[1]).max() > 2e-5
    scale = np.abs(S.zeta[1]).max() * np.sum(1.0 / (G["pm"] * G["pn"]))
    assert abs(ro.volume(G, S.zeta[1]) - v0) <= 1e-12 * scale


def _amplification(a):
    """Largest |eigenvalue| of one substep of the scheme for the linear 1D wave equation on a
    staggered grid, worst-resolved mode, effective Courant number a = 2 c dt / dx."""
    def step(x):
        zb, zn, ub, un, rzb, rub = x
        Rz = lambda u: -1j * a * u
        Ru = lambda z: -1j * a * z
        rz = Rz(un)
        zs = zb + 2 * rz
        ru = Ru(0.68 * zn + 0.16 * (zb + zs))
        us = ub + 2 * ru
        znew = zn + (5 / 12 * Rz(us) + 8 / 12 * rz - 1 / 12 * rzb)
        unew = un + (5 / 12 * Ru(0.6 * znew + 0.4 * zs) + 8 / 12 * ru - 1 / 12 * rub)
        return np.array([zn, znew, un, unew, rz, ru])
    M = np.array([step(e) for e in np.eye(6, dtype=complex)]).T
    return max(abs(np.linalg.eigvals(M)))


def test_oracle_stability_limit_matches_the_von_neumann_analysis():
    # the analysis: stable up to an effective Courant number of ~2.14 (1D); on a square grid
    # the worst mode has a = 2 sqrt(2) c dt / dx, so c dt / dx < 2.14 / (2 sqrt 2) = 0.757
    a_lim = next(a for a in np.arange(1.5, 3.0, 0.01) if _amplification(a) > 1.0 + 1e-9)
    alpha = a_lim / (2.0 * np.sqrt(2.0))
    assert 0.74 < alpha < 0.77
    cfg, g, G = _basin(40, 40, f=False)
    c = np.sqrt(10.0 * 4000.0)
    bump = 0.1 * np.exp(-((g.x - g.x.mean()) ** 2 + (g.y - g.y.mean()) ** 2) / (30e3) ** 2)
    zero = np.zeros_like(bump)

    def run(courant):
        S = ro.State(g.J, g.I)
        S.zeta[1][...] = bump
        ro._ring(S.zeta[1])
        with np.errstate(all="ignore"):
            ro.main2d(G, S, 800, courant * 5e3 / c, zero, zero, 0.0)
        return np.nanmax(np.abs(S.zeta[1])) if np.isfinite(S.zeta[1]).all() else np.inf

    assert run(0.93 * alpha) < 0.2          # stable just below the analysed limit
    assert run(1.07 * alpha) > 1e3          # unstable just above it


def _gpu_model(G, g, cfg, precision, su, sv, rdrag2, N=5, ndtfast=1):
    from sailfish_b200.model import Model
    m = Model(g, cfg["boundary"], cfg["dt"], ndtfast, precision=precision, semantics="roms")
    m.set_forcing(su, sv, rdrag2)
    return m


def _model_2d(m):
    """(zeta, ubar, vbar) slots [n-1, n] and the averages of a model, as host FP64 arrays."""
    sh = (m.grid.J, m.grid.I)
    out = {}
    for n in ("zeta", "ubar", "vbar", "rzeta", "rubar", "rvbar"):
        buf = getattr(m, n).double().cpu().numpy()
        out[n] = [buf[m.slots[k]].reshape(sh) for k in range(2)]
    for n in ("Zt_avg1", "DU_avg1", "DV_avg1", "DU_avg2", "DV_avg2"):
        out[n] = getattr(m, n).double().cpu().numpy().reshape(sh)
    return out


@pytest.mark.gpu
def test_cuda_2d_steps_bit_exact_against_the_oracle():
    import torch
    cfg, g, G = _basin(60, 44, dx=5e3)
    su = _wind(g)
    sv = 0.25 * su
    m = _gpu_model(G, g, cfg, "fp64", su, sv, 3e-3)
    bump = 0.05 * np.exp(-((g.x - g.x.mean() * 0.7) ** 2 + (g.y - g.y.mean()) ** 2) / (40e3) ** 2)
    S = ro.State(g.J, g.I)
    S.zeta[1][...] = bump
    ro._ring(S.zeta[1])
    init = np.zeros((3,) + S.zeta[1].shape)
    init[m.slots[1]] = S.zeta[1]
    m.load({"zeta": init})
    dt = 15.0
    m.dtfast = dt
    m.step2d(60)
    torch.cuda.synchronize()
    ro.main2d(G, S, 60, dt, su, sv, 3e-3)
    out = _model_2d(m)
    for n in ("zeta", "ubar", "vbar"):
        for k in range(2):
            np.testing.assert_array_equal(out[n][k], getattr(S, n)[k], err_msg="%s[%d]" % (n, k))
    assert np.abs(out["vbar"][1]).max() > 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("ndtfast", [10, 30])
def test_cuda_barotropic_loop_bit_exact_against_the_oracle(ndtfast):
    """nfast+1 substeps with the fast-time averages (Zt_avg1, DU/DV_avg1, DU/DV_avg2)."""
    import ctypes
    import torch
    from sailfish_b200 import host
    cfg, g, G = _basin(50, 50, dx=2e3, h=200.0)     # c dtfast / dx <= 0.54 (stable)
    su = _wind(g, 0.15)
    sv = -0.2 * su
    m = _gpu_model(G, g, cfg, "fp64", su, sv, 3e-3, ndtfast=ndtfast)
    m.dtfast = 240.0 / ndtfast
    rng = np.random.default_rng(ndtfast)
    S = ro.State(g.J, g.I)
    S.zeta[1][...] = 0.02 * np.exp(-((g.x - g.x.mean()) ** 2 + (g.y - g.y.mean()) ** 2) / (20e3) ** 2)
    ro._ring(S.zeta[1])
    S.ubar[1][1:-1, 2:-1] = 0.01 * rng.standard_normal((g.J - 2, g.I - 3))
    init = {n: np.zeros((3, g.J, g.I)) for n in ("zeta", "ubar")}
    init["zeta"][m.slots[1]] = S.zeta[1]
    init["ubar"][m.slots[1]] = S.ubar[1]
    m.load(init)
    nfast, w1, _ = host.set_weights(ndtfast)
    W1, W2 = ro.roms_weights(nfast, w1)
    np.testing.assert_array_equal(W1, m.W1)
    np.testing.assert_array_equal(W2, m.W2)
    for _ in range(2):
        s = m.state2d()
        m._roms_loop(s, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        m._sync_slots(s)
        ro.barotropic_loop(G, S, nfast, W1, W2, m.dtfast, su, sv, 3e-3)
    torch.cuda.synchronize()
    out = _model_2d(m)
    for n in ("zeta", "ubar", "vbar", "rzeta", "rubar", "rvbar"):
        for k in range(2):
            np.testing.assert_array_equal(out[n][k], getattr(S, n)[k], err_msg="%s[%d]" % (n, k))
    for n in ("Zt_avg1", "DU_avg1", "DV_avg1", "DU_avg2", "DV_avg2"):
        np.testing.assert_array_equal(out[n], getattr(S, n), err_msg=n)
    assert np.abs(out["DV_avg2"]).max() > 0


@pytest.mark.gpu
def test_fp32_loop_against_fp64():
    import ctypes
    import torch
    cfg, g, G = _basin(120, 120, dx=2e3, h=1000.0)   # c dtfast / dx = 0.4
    su = _wind(g, 0.15)
    sv = 0.1 * su
    res = {}
    for prec in ("fp64", "fp32"):
        m = _gpu_model(G, g, cfg, prec, su, sv, 3e-3, ndtfast=30)
        m.dtfast = 240.0 / 30
        z = np.zeros((3, g.J, g.I))
        z[m.slots[1]] = 0.05 * np.exp(-((g.x - g.x.mean()) ** 2 + (g.y - g.y.mean()) ** 2) / (30e3) ** 2)
        m.load({"zeta": z})
        for _ in range(5):
            s = m.state2d()
            m._roms_loop(s, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
            m._sync_slots(s)
        torch.cuda.synchronize()
        res[prec] = _model_2d(m)
    # relative to each field's largest magnitude: FP32 stencils, FP64 averages
    for n, tol in (("zeta", 2e-5), ("ubar", 1e-4), ("vbar", 1e-4)):
        a, b = res["fp64"][n][1], res["fp32"][n][1]
        assert np.abs(b - a).max() <= tol * np.abs(a).max(), n
    for n, tol in (("Zt_avg1", 2e-5), ("DU_avg1", 1e-4), ("DV_avg2", 1e-4)):
        a, b = res["fp64"][n], res["fp32"][n]
        assert np.abs(b - a).max() <= tol * np.abs(a).max(), n


# ---- the baroclinic step in ROMS form ----------------------------------------------------------
def _case3d(Lm=24, Mm=16, N=6, dx=2e3, dt=120.0, ndtfast=20, tau0=0.1):
    """A closed shelf basin with one seamount (depth 50..4000 m, c dtfast / dx <= 0.6), wind
    tau0 cos(pi y / Ly) and a 5 cm surface bump, as (cfg, oracle grid, oracle boundary lists,
    oracle state, sustr, svstr)."""
    import oracle as orc
    from golden_io import BND_KEYS
    from sailfish_b200 import configs
    cfg = configs.basin(Lm, Mm, N, dx, [(0.5, 0.6)], dt=dt, ndtfast=ndtfast)
    g, B = cfg["grid"], cfg["boundary"]
    og = orc.Grid(g.L, g.M, g.N, g.h, g.pm, g.pn, g.on_u, g.om_v, g.fomn, g.sc_r, g.sc_w,
                  g.Cs_r, g.Cs_w, g.hc, g.Vtransform)
    bd = {}
    for name in ("zetaBC", "ubarBC", "vbarBC", "uvelBC", "vvelBC"):
        for f in ("bcIdx", "bcIdx1", "bcIdx2", "bcIdxFieldIdx2", "bcIdxFieldType", "LBC"):
            bd["%s_%s" % (name, f)] = getattr(getattr(B, name), f)
    for f in BND_KEYS:
        bd[f] = getattr(B, f)
    st = ro.State3D(og)
    st.S.Zt_avg1[...] = 0.05 * np.exp(-((g.x - 0.4 * g.x.max()) ** 2 + (g.y - g.y.mean()) ** 2)
                                      / (8.0 * dx) ** 2)
    su = _wind(g, tau0)
    sv = 0.2 * su
    return cfg, og, orc.Boundary(bd), st, su, sv


def _run_oracle3d(cfg, og, B, st, su, sv, nsteps, rdrag2=3e-3, on_step=None):
    from sailfish_b200 import host
    nfast, w1, _ = host.set_weights(cfg["ndtfast"])
    W1, W2 = ro.roms_weights(nfast, w1)
    with np.errstate(all="raise"):
        ro.main3d(og, B, st, nsteps, cfg["dt"], cfg["ndtfast"], nfast, W1, W2, su, sv, rdrag2,
                  on_step=on_step)


def test_oracle_3d_conserves_volume_and_couples_the_depth_mean():
    """ROMS-form baroclinic steps with wind, drag and Coriolis over a seamount: the volume of
    the fast-time mean surface is conserved, the 3D velocity's depth mean equals the barotropic
    velocity the next loop starts from (the coupling step3d_uv makes), and the flow stays
    bounded and wind-driven."""
    cfg, og, B, st, su, sv = _case3d()
    g = cfg["grid"]
    G = dict(pm=g.pm, pn=g.pn)
    v0 = ro.volume(G, st.S.Zt_avg1)
    _run_oracle3d(cfg, og, B, st, su, sv, 12)
    S, O, N, J, I = st.S, st.O, og.N, og.J, og.I
    scale = np.abs(S.Zt_avg1).max() * np.sum(1.0 / (g.pm * g.pn))
    assert abs(ro.volume(G, S.Zt_avg1) - v0) <= 1e-12 * scale
    u = O.t3("u").reshape(N + 1, J, I)[:N]
    Hz = og.Hz.reshape(N, J, I)
    hzu = 0.5 * (Hz[:, :, 1:] + Hz[:, :, :-1])
    mean = (hzu * u[:, :, 1:]).sum(0) / hzu.sum(0)
    inner = (slice(2, J - 2), slice(2, I - 3))        # U faces i = 3..I-3 (mean[.., i-1])
    np.testing.assert_allclose(mean[inner], S.ubar[1][2:J - 2, 3:I - 2], rtol=0,
                               atol=1e-12 * np.abs(S.ubar[1]).max())
    assert 1e-4 < np.abs(u).max() < 1.0
    # relative to the depth mean, the surface layer moves downwind: east in the south, where
    # tau_x = tau0 cos(pi y / Ly) > 0, west in the north
    shear = u[N - 1, :, 1:] - mean
    assert shear[J // 4, 2:I - 3].mean() > 0 > shear[3 * J // 4, 2:I - 3].mean()


def _roms_model3d(cfg, st, su, sv, precision, rdrag2=3e-3):
    from sailfish_b200.model import Model
    m = Model(cfg["grid"], cfg["boundary"], cfg["dt"], cfg["ndtfast"], precision=precision,
              semantics="roms")
    m.set_forcing(su, sv, rdrag2)
    m.load({"Zt_avg1": np.array(st.S.Zt_avg1)})
    return m


@pytest.mark.gpu
def test_cuda_3d_steps_bit_exact_against_the_oracle():
    """Four ROMS-form baroclinic steps (Euler, AB2, then AB3 over the three right-hand sides)
    over a seamount with wind, drag and Coriolis: the FP64 CUDA path and the oracle, bit for
    bit, including the three right-hand-side slots."""
    import torch
    cfg, og, B, st, su, sv = _case3d(40, 28, 8)
    m = _roms_model3d(cfg, st, su, sv, "fp64")
    m.step(4)
    torch.cuda.synchronize()
    _run_oracle3d(cfg, og, B, st, su, sv, 4)
    s = m.state()
    S, O = st.S, st.O
    sh = (og.J, og.I)
    for n in ("zeta", "ubar", "vbar"):
        for k in range(2):
            np.testing.assert_array_equal(s[n][s["slots"][k]].reshape(sh), getattr(S, n)[k],
                                          err_msg="%s[%d]" % (n, k))
    for n in ("Zt_avg1", "DU_avg1", "DV_avg1"):
        np.testing.assert_array_equal(s[n].reshape(sh), getattr(S, n), err_msg=n)
    for n in ("u", "v"):
        np.testing.assert_array_equal(s[n].reshape(-1), O.t3(n), err_msg=n)
    for k in range(3):      # the right-hand sides of the last three steps, newest first
        np.testing.assert_array_equal(m._ru3[k].cpu().numpy().reshape(-1), st.ru3[k], err_msg="ru%d" % k)
        np.testing.assert_array_equal(m._rv3[k].cpu().numpy().reshape(-1), st.rv3[k], err_msg="rv%d" % k)
    np.testing.assert_array_equal(s["W"].reshape(-1), O.W.reshape(-1), err_msg="W")
    assert np.abs(O.t3("v")).max() > 1e-4


@pytest.mark.gpu
def test_cuda_3d_fp32_against_fp64():
    """20 ROMS-form steps at 160 x 96 x 16: FP32 stencils with FP64 fast-time averages and
    depth sums against FP64, relative to each field's largest magnitude."""
    import torch
    res = {}
    for prec in ("fp64", "fp32"):
        cfg, og, B, st, su, sv = _case3d(160, 96, 16)
        m = _roms_model3d(cfg, st, su, sv, prec)
        m.step(20)
        torch.cuda.synchronize()
        res[prec] = m.state()
    a, b = res["fp64"], res["fp32"]
    for n, tol in (("Zt_avg1", 1e-4), ("u", 1e-3), ("v", 1e-3)):
        x, y = a[n].reshape(-1), b[n].reshape(-1)
        assert np.isfinite(y).all(), n
        assert np.abs(y - x).max() <= tol * np.abs(x).max(), (n, np.abs(y - x).max() / np.abs(x).max())
