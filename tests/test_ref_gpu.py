"""The reference's own CUDA kernels on the GPU (baseline/ref_gpu.py, the plain FP64 step the
benchmark compares with): NVRTC builds them with the reference's options, and the launcher
runs them in main3d order.  Built without FMA contraction they reproduce the reference's
golden main3d runs and this package's FP64 path, which pins the launcher (launch geometry,
argument order, slot rotation, boundary scatters), except where the reference's own GPU code
races: its zetabc copyBC launch (modules/mod_BC.c:16-21) has two entries writing each corner
node of the ring and entries whose source node another entry of the same launch writes, so on
the GPU the four corners take whichever write lands last, while the golden runs (threads in
order on the host) and this package (the launches' sequential effect, resolved on the host)
take the sequential one.  Those nodes differ; everything else agrees bit for bit after one
step, and to a small fraction of the field's scale after the corners' values have spread
(the reference's step amplifies them)."""
import os
import sys

import numpy as np
import pytest

from golden_io import load, boundary_dict

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "baseline"))
import ref_gpu  # noqa: E402

NAMES2 = ("zeta", "ubar", "vbar", "rzeta", "rubar", "rvbar")
needs_src = pytest.mark.skipif(not ref_gpu.available(),
                               reason="baseline/_ref/src not generated (no reference checkout)")


@needs_src
def test_nvrtc_builds_every_module_for_sm100a():
    out = ref_gpu.cubins(fmad=True)
    assert set(out) == set(ref_gpu.MODULES)
    assert all(len(c) > 1000 for c in out.values())


def _golden_ref(tag):
    d = load("main3d_%s.npz" % tag)
    g = lambda k: d["in_grid_" + k]
    b = dict(L=int(d["in_L"]), M=int(d["in_M"]), N=int(d["in_N"]), hc=float(g("hc")),
             Vtransform=int(d["in_Vtransform"]), dt=float(d["in_dt"]),
             ndtfast=int(d["in_ndtfast"]), lists=boundary_dict(d, "in_bnd_"))
    for k in ("h", "pm", "pn", "on_u", "om_v", "fomn", "sc_r", "sc_w", "Cs_r", "Cs_w"):
        b[k] = g(k)
    init = {n: d["in_" + n] for n in NAMES2 + ("W", "Huon", "Hvom", "Zt_avg1", "DU_avg1",
                                               "DV_avg1", "AKv")}
    for n in ("u", "v", "ru", "rv"):
        init[n] = d["in_" + n][2]
    return d, b, init


@pytest.mark.gpu
@needs_src
@pytest.mark.parametrize("tag", ["square", "nonsquare", "vt1"])
def test_reference_kernels_on_the_gpu_reproduce_the_golden_runs(tag):
    import torch
    d, b, init = _golden_ref(tag)
    r = ref_gpu.RefGPU(b, int(d["in_nfast"]), d["in_w1"], d["in_w2"], fmad=False, init=init)
    r.step(int(d["in_nsteps"]), AK=float(d["in_AK"]))
    torch.cuda.synchronize()
    for n in NAMES2:
        assert r.slots[n] == list(d["out_slots_" + n]), n
        _close(getattr(r, n).cpu().numpy(), d["out_" + n].reshape(-1), n)
    for n in ("u", "v"):
        _close(r.t3(n).cpu().numpy(), d["out_" + n][2].reshape(-1), n)
    # ru, rv are the right-hand side evaluated from those u, v (differences of neighbours,
    # times the fluxes): the corners' perturbation shows in them a few times larger
    for n in ("ru", "rv"):
        _close(r.t3(n).cpu().numpy(), d["out_" + n][2].reshape(-1), n, tol=1e-2)
    for n in ("W", "Zt_avg1", "DU_avg1", "DV_avg1", "z_w", "z_r", "Hz"):
        _close(getattr(r, n).cpu().numpy(), d["out_" + n].reshape(-1), n)


def _close(a, b, name, tol=1e-3):
    """Equal where finite up to tol of the field's largest finite magnitude (the corner race of
    the reference's GPU boundary scatter spreads over the golden runs' three steps)."""
    fin = np.isfinite(b)
    assert np.array_equal(fin, np.isfinite(a)), name
    scale = max(np.abs(b[fin]).max() if fin.any() else 0.0, 1e-300)
    assert np.abs(a[fin] - b[fin]).max() <= tol * scale, (name, np.abs(a[fin] - b[fin]).max() / scale)


@pytest.mark.gpu
@needs_src
def test_reference_kernels_match_the_fp64_path_on_a_larger_basin():
    """64 x 64 x 8 basin from a 1 mm surface bump, 1 step (the reference's step grows the bump
    by orders of magnitude per step): the reference's kernels (no FMA contraction) and this
    package's FP64 path, bit for bit."""
    import torch
    from sailfish_b200 import configs, host
    from sailfish_b200.model import Model
    cfg = configs.basin(64, 64, 8, 2.0e3, [(0.5, 0.6)], dt=240.0, ndtfast=20)
    g, B = cfg["grid"], cfg["boundary"]
    bump = 1e-3 * np.exp(-((g.x - g.x.max() / 2) ** 2 + (g.y - g.y.max() / 3) ** 2) / (2e4) ** 2)
    m = Model(g, B, cfg["dt"], cfg["ndtfast"], precision="fp64")
    m.Zt_avg1.copy_(torch.from_numpy(bump.ravel()))
    m.step(1)
    torch.cuda.synchronize()
    s = m.state()
    lists = {}
    for name in ("zetaBC", "ubarBC", "vbarBC", "uvelBC", "vvelBC"):
        for f in ("bcIdx", "bcIdx1", "bcIdx2", "bcIdxFieldIdx2", "bcIdxFieldType", "LBC"):
            lists["%s_%s" % (name, f)] = getattr(getattr(B, name), f)
    for f in ("zetaClosedOrGradientBCIdx1", "zetaClosedOrGradientBCIdx2", "zetaClampedBCIdx1",
              "ubarClosedBCIdx1", "vbarClosedBCIdx1", "ubarClampedBCIdx1", "vbarClampedBCIdx1",
              "ubarGradientBCIdx1", "ubarGradientBCIdx2", "vbarGradientBCIdx1", "vbarGradientBCIdx2"):
        lists[f] = getattr(B, f)
    b = dict(L=g.L, M=g.M, N=g.N, hc=g.hc, Vtransform=g.Vtransform, dt=cfg["dt"],
             ndtfast=cfg["ndtfast"], lists=lists)
    for k in ("h", "pm", "pn", "on_u", "om_v", "fomn", "sc_r", "sc_w", "Cs_r", "Cs_w"):
        b[k] = getattr(g, k)
    nf, w1, w2 = host.set_weights(cfg["ndtfast"])
    r = ref_gpu.RefGPU(b, nf, w1, w2, fmad=False, init={"Zt_avg1": bump.ravel()})
    r.step(1)
    torch.cuda.synchronize()
    # after one step only the ring's four corners (and what they feed within the step) can
    # differ: compare bit for bit away from them
    J, I = g.J, g.I
    jj, ii = np.meshgrid(np.arange(J), np.arange(I), indexing="ij")
    far = ((np.minimum(ii, I - 1 - ii) > 3) | (np.minimum(jj, J - 1 - jj) > 3)).reshape(-1)
    for n in ("zeta", "ubar", "vbar"):
        a = np.stack([getattr(r, n).cpu().numpy().reshape(3, -1)[r.slots[n][k]] for k in range(3)])
        c = np.stack([s[n][s["slots"][k]].reshape(-1) for k in range(3)])
        assert np.isfinite(c).all()
        np.testing.assert_array_equal(c[:, far], a[:, far], err_msg=n)
    far3 = np.tile(far, g.N + 1)
    for n in ("u", "v"):
        np.testing.assert_array_equal(s[n].reshape(-1)[far3], r.t3(n).cpu().numpy()[far3], err_msg=n)
    for n, m_ in (("W", far3), ("Zt_avg1", far), ("DU_avg1", far), ("z_w", far3),
                  ("Hz", np.tile(far, g.N))):
        np.testing.assert_array_equal(s[n].reshape(-1)[m_], getattr(r, n).cpu().numpy()[m_],
                                      err_msg=n)
