"""Learned closure in the time step: fused inference against the NumPy oracle, the
column-selected GLS and the range mask it relies on, and training on plain-GLS data with a
held-out measure of what the trained network gains over the method without it."""
import ctypes

import numpy as np
import pytest
import torch

import mlp_oracle as mo


def test_normalisation_folds_into_first_layer():
    from sailfish_b200 import closure
    net = closure.Network(32, seed=3, device="cpu")
    nf = closure.nfeat(32)
    rng = np.random.default_rng(0)
    X = torch.tensor(rng.standard_normal((500, 128)) * 3.0 + 5.0, dtype=torch.float32)
    X[:, nf:] = 0.0
    net.fit_normalisation(X)
    W0 = net.W[0] * net.isd[None, :]
    b0 = net.b[0] - W0 @ net.mu
    folded = X @ W0.T + b0
    direct = ((X - net.mu) * net.isd) @ net.W[0].T + net.b[0]
    torch.testing.assert_close(folded, direct, rtol=1e-4, atol=1e-3)
    assert torch.all(net.lo[:nf] < X.min(0).values[:nf])
    assert torch.all(net.hi[:nf] > X.max(0).values[:nf])


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _st():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["gelu", "relu"])
@pytest.mark.parametrize("n", [128, 300, 4096 + 77])
def test_fused_inference_matches_oracle(n, kind):
    from sailfish_b200._lib import MLP_ACT, MlpParams, lib
    rng = np.random.default_rng(n)
    W = [mo.bf16(rng.standard_normal((128, 128)) / np.sqrt(128)) for _ in range(5)]
    b = [rng.standard_normal(128) * 0.05 for _ in range(5)]
    X = rng.standard_normal((n, 128)).astype(np.float32)
    tW = [torch.tensor(w, dtype=torch.bfloat16, device="cuda") for w in W]
    tb = [torch.tensor(v, dtype=torch.float32, device="cuda") for v in b]
    P = MlpParams()
    for l in range(5):
        P.W[l], P.b[l] = tW[l].data_ptr(), tb[l].data_ptr()
    P.act = MLP_ACT[kind]
    tX = torch.tensor(X, device="cuda")
    Y = torch.full((n, 128), float("nan"), device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.sf_mlp_infer(ctypes.byref(P), n, _p(tX), _p(Y), _p(err), _st()) == 0, \
        lib.sf_mlp_last_error()
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref, _, _ = mo.forward(W, b, X, kind)
    got = Y.cpu().numpy()
    assert np.isfinite(got).all()
    # BF16 activations between layers; the hardware tanh differs from tanhf by ~2^-11
    np.testing.assert_allclose(got, ref, rtol=0, atol=2e-2 * np.abs(ref).max())


def _gls_setup(precision="fp32"):
    from sailfish_b200 import closure, configs
    from sailfish_b200.model import Model
    cfg = configs.small(24, 16, 12)
    m = Model(cfg["grid"], cfg["boundary"], cfg["dt"], cfg["ndtfast"], precision=precision)
    m.start()
    cols = closure.Columns(m)
    closure.wind_driven_state(m, cols, 0.1, 0.3, 500.0, np.random.default_rng(1))
    return m, cols


@pytest.mark.gpu
def test_analytic_bvf():
    from sailfish_b200 import closure
    m, cols = _gls_setup("fp64")
    torch.cuda.synchronize()
    zw = m.z_w.cpu().numpy()
    ref = closure.G * closure.ALPHA * (20.0 / 500.0) * np.exp(zw / 500.0)
    np.testing.assert_allclose(cols.bvf.cpu().numpy(), ref, rtol=1e-12)


@pytest.mark.gpu
def test_gls_on_selected_columns_only():
    m, cols = _gls_setup()
    s2 = m.grid.s2
    sel = torch.zeros(s2, dtype=torch.uint8, device="cuda")
    sel[::3] = 1
    names = ("tke", "gls", "Akt", "Akk", "Akp", "Lscale")
    snap = {k: getattr(cols, k).clone() for k in names}
    akv0 = m.AKv.clone()
    cols.gls_step()                      # all columns
    full = {k: getattr(cols, k).clone() for k in names}
    akv_full = m.AKv.clone()
    for k, v in snap.items():
        getattr(cols, k).copy_(v)
    m.AKv.copy_(akv0)
    cols.gls_step(sel)                   # selected columns only
    torch.cuda.synchronize()
    on = sel.bool()
    for k in names:
        got = getattr(cols, k).reshape(-1, s2)
        torch.testing.assert_close(got[:, on], full[k].reshape(-1, s2)[:, on], rtol=0, atol=0)
        torch.testing.assert_close(got[:, ~on], snap[k].reshape(-1, s2)[:, ~on], rtol=0, atol=0)
    torch.testing.assert_close(m.AKv.reshape(-1, s2)[:, on], akv_full.reshape(-1, s2)[:, on],
                               rtol=0, atol=0)


def _range_mask_case():
    from sailfish_b200 import closure
    from sailfish_b200._lib import lib, check
    m, cols = _gls_setup()
    g = m.grid
    X = torch.zeros((g.s2, 128), device="cuda")
    cols.features(X)
    lo = torch.full((128,), -1e30, device="cuda")
    hi = torch.full((128,), 1e30, device="cuda")
    nf = closure.nfeat(g.N)
    kd = nf - 1                                     # depth feature: only the deepest columns
    lo[kd] = float(X[:, kd].max().item()) - 0.01
    mask = torch.full((g.s2,), 7, dtype=torch.uint8, device="cuda")
    check(lib.sf_closure_range_mask(m.ctx.ptr, _p(X), nf, _p(lo), _p(hi), _p(mask),
                                    _st()), "sf_closure_range_mask")
    torch.cuda.synchronize()
    Xh = X.cpu().numpy()
    idx = np.arange(g.s2)
    i, j = idx % g.I, idx // g.I
    interior = (i != 0) & (i != g.I - 1) & (j != 0) & (j != g.J - 1)
    inside = np.all((Xh[:, :nf] >= lo.cpu().numpy()[:nf]) &
                    (Xh[:, :nf] <= hi.cpu().numpy()[:nf]), axis=1)
    expect = (interior & ~inside).astype(np.uint8)
    return mask.cpu().numpy(), expect


@pytest.mark.gpu
def test_closure_range_mask_flags_out_of_range_columns():
    got, expect = _range_mask_case()
    np.testing.assert_array_equal(got, expect)
    assert 0 < expect.sum() < expect.size


@pytest.mark.gpu
def test_trained_network_gains_over_the_method_without_it():
    """Train on plain-GLS runs of a small basin, evaluate on a held-out run (other wind and
    stratification): the trained network's Akv/Akt log10 RMS error against GLS must be well
    below that of the reference's own method (constant AKv = 1e-3 m2/s, Akt = 1e-6 m2/s
    background) and of the untrained network."""
    from sailfish_b200 import closure, configs
    cfg = configs.small(48, 32, 16)
    N = cfg["grid"].N
    # every run spans the wind and stratification ranges across its basin
    X, T = closure.generate(cfg, runs=6, spin=20, keep=3, every=4, seed=11, pattern=True,
                            spread=True)
    Xv, Tv = closure.generate(cfg, runs=2, spin=20, keep=2, every=4, seed=99, pattern=True,
                              spread=True)
    net = closure.Network(N, seed=0)
    net.fit_normalisation(X)
    Y0 = net.infer(Xv)
    e0 = closure.log_rms(Y0, Tv, N)
    hist = net.train(X, T, steps=1500, batch=1024, lr=2e-3, log_every=500)
    Y = net.infer(Xv)
    e = closure.log_rms(Y, Tv, N)
    const = torch.zeros_like(Tv)
    const[:, :N - 1] = -3.0                 # log10(1e-3), modules/mod_ocean.py:91
    const[:, N - 1:2 * (N - 1)] = -6.0      # log10(1e-6)
    ec = closure.log_rms(const, Tv, N)
    print("held-out log10 RMS (Akv, Akt): trained", e, "untrained", e0, "constant", ec,
          "loss", hist)
    assert hist[-1][1] < 0.2 * hist[0][1]
    assert e[0] < 0.5 * ec[0] and e[1] < 0.5 * ec[1]
    assert e[0] < 0.5 * e0[0] and e[1] < 0.5 * e0[1]


@pytest.mark.gpu
def test_closure_in_the_time_step_with_fallback():
    """'mlp' closure with a range that excludes some columns: those get plain GLS exactly,
    the others the network's clipped coefficients."""
    from sailfish_b200 import closure, configs
    from sailfish_b200.model import Model
    cfg = configs.small(24, 16, 12)
    N = cfg["grid"].N
    X, T = closure.generate(cfg, runs=2, spin=10, keep=2, every=2, seed=5)
    net = closure.Network(N, seed=1)
    net.fit_normalisation(X)
    net.train(X, T, steps=100, batch=256)
    kd = closure.nfeat(N) - 1
    net.lo.fill_(-1e30)                                 # every column in range ...
    net.hi.fill_(1e30)
    net.hi[kd] = float(X[:, kd].max().item()) - 0.05    # ... except the deepest: plain GLS

    def make():
        m = Model(cfg["grid"], cfg["boundary"], cfg["dt"], cfg["ndtfast"], precision="fp32")
        m.start()
        return m
    m1, m2 = make(), make()
    c_mlp = closure.Closure(m1, "mlp", net)
    c_gls = closure.Closure(m2, "gls")
    for m, c in ((m1, c_mlp), (m2, c_gls)):
        closure.wind_driven_state(m, c.cols, 0.1, 0.5, 400.0, np.random.default_rng(3))
        m.AKv.fill_(1e-5)
        c()
    torch.cuda.synchronize()
    mask = c_mlp.mask.bool()
    assert 0 < int(mask.sum()) < mask.numel()
    s2 = m1.grid.s2
    a1, a2 = m1.AKv.reshape(N + 1, s2), m2.AKv.reshape(N + 1, s2)
    torch.testing.assert_close(a1[:, mask], a2[:, mask], rtol=0, atol=0)
    g = m1.grid
    idx = torch.arange(s2, device="cuda")
    i, j = idx % g.I, idx // g.I
    inner = (i != 0) & (i != g.I - 1) & (j != 0) & (j != g.J - 1) & ~mask
    v = a1[1:N][:, inner]
    assert torch.isfinite(v).all()
    assert float(v.min()) >= 1e-6 * (1 - 1e-6) and float(v.max()) <= 1e-1 * (1 + 1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_fused_closure_step_matches_the_composition(precision):
    """sf_closure_step against features -> range mask -> sf_mlp_infer -> sf_closure_apply."""
    from sailfish_b200 import closure, configs
    from sailfish_b200.model import Model
    cfg = configs.small(40, 24, 14)
    N = cfg["grid"].N
    X, T = closure.generate(cfg, runs=2, spin=8, keep=2, every=2, seed=21)
    net = closure.Network(N, seed=2)
    net.fit_normalisation(X)
    net.train(X, T, steps=200, batch=512)
    kd = closure.nfeat(N) - 1
    net.hi[kd] = float(X[:, kd].max().item()) - 0.05

    out = []
    for fused in (True, False):
        m = Model(cfg["grid"], cfg["boundary"], cfg["dt"], cfg["ndtfast"], precision=precision)
        m.start()
        c = closure.Closure(m, "mlp", net, fused=fused)
        closure.wind_driven_state(m, c.cols, 0.12, 1.0, 600.0, np.random.default_rng(4))
        m.AKv.fill_(2e-5)
        c.cols.Akt.fill_(3e-6)
        c()
        torch.cuda.synchronize()
        out.append((c.mask.clone(), m.AKv.clone(), c.cols.Akt.clone()))
    (mf, af, tf), (mu, au, tu) = out
    assert torch.equal(mf, mu)
    assert 0 < int(mf.sum()) < mf.numel()
    # identical features and BF16 operands; the tile epilogues round the same way
    torch.testing.assert_close(af, au, rtol=1e-3, atol=0)
    torch.testing.assert_close(tf, tu, rtol=1e-3, atol=0)


@pytest.mark.gpu
def test_training_snapshots_from_roms_form_runs():
    """closure.generate_roms: snapshots along ROMS-form runs from rest with plain GLS, one per
    `every` steps after the spin-up, every row finite, targets log10 Akv/Akt inside the clip
    range [-6, -1] and varying (the turbulence develops along the run)."""
    from sailfish_b200 import closure, configs
    cfg = configs.basin(48, 32, 8, 2.0e3, [(0.5, 0.6)], dt=240.0, ndtfast=30)
    X, T = closure.generate_roms(cfg, runs=2, hours=4.0, spin_hours=2.0, every=10, seed=3,
                                 gls_model="k-psi")
    N = cfg["grid"].N
    nc = 48 * 32
    assert X.shape[0] == 2 * 3 * nc and T.shape == X.shape          # snapshots at 30, 40, 50
    assert bool(torch.isfinite(X).all()) and bool(torch.isfinite(T).all())
    t = T[:, :2 * (N - 1)]
    assert float(t.min()) >= -6.0 - 1e-6 and float(t.max()) <= -1.0 + 1e-6
    assert float(t[:, :N - 1].std()) > 0.05
