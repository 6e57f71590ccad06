"""Learned vertical-mixing closure: training data from plain GLS runs, training on the GPU with
the library's own tensor-core forward/backward kernels, and the per-step closure with plain
GLS as the fallback for columns outside the training range.

The reference's time step keeps its viscosity AKv at the constant 1e-3 m2/s of
modules/mod_ocean.py:91 (its GLS closure, nonlinear/gls_corrector_step.py, is untranslated
ROMS Fortran).  Plain GLS (sf_gls_corrector) is this package's closure; the network stands in
for its Akv/Akt at a fraction of the cost, and its error is measured against GLS.

Rows: one water column each, 128 FP32 features from sf_closure_features; with nl = N-1
interior W levels: log10 shear^2 in [0, nl), signed log N^2 in [nl, 2nl), then log10 surface
friction velocity squared, surface buoyancy flux and log10 depth.  Targets: log10 Akv at
levels 1..N-1 in outputs [0, nl), log10 Akt in [nl, 2nl).  A network serves one N (N <= 63).
"""
import ctypes
import math

import numpy as np
import torch

from . import configs
from ._lib import MLP_ACT, GlsParams, MlpParams, check, lib
from .model import Model, stream_handle

LAYERS, WIDTH = 5, 128


def nfeat(N):
    """Features used of the 128 for N levels: two per interior W level, three scalars."""
    return 2 * (N - 1) + 3


def nout(N):
    """Outputs trained for N levels: Akv and Akt at each interior W level."""
    return 2 * (N - 1)


RHO0 = 1025.0        # modules/mod_constants.py:25
G = 10.0             # modules/mod_constants.py:26
ALPHA = 1.7e-4       # linear EOS thermal expansion, utility/test.in:453


_GLS_BASE = dict(Kmin=7.6e-6, Pmin=1.0e-12, Akv_bak=1.0e-5, Akt_bak=1.0e-6, Akk_bak=5.0e-6,
                 Akp_bak=5.0e-6, Zos=0.02, Zob=0.02, rdrag2=3.0e-3)
# Members of the GLS family (psi = cmu0^p k^m l^n), with the floors and backgrounds above:
# k-epsilon as the reference's input file selects it (utility/test.in:355-367); k-omega and the
# generic k-psi model of Umlauf and Burchard (2003) ("gen": p = 2, m = 1, n = -0.67) with the
# constants of Warner et al. (2005, Ocean Modelling 8, Table 1).
GLS_PRESETS = {
    "k-epsilon": dict(p=3.0, m=1.5, n=-1.0, cmu0=0.5477, c1=1.44, c2=1.92, c3m=-0.4, c3p=1.0,
                      sigk=1.0, sigp=1.30),
    "k-omega": dict(p=-1.0, m=0.5, n=-1.0, cmu0=0.5477, c1=0.555, c2=0.833, c3m=-0.6, c3p=1.0,
                    sigk=2.0, sigp=2.0),
    "gen": dict(p=2.0, m=1.0, n=-0.67, cmu0=0.5544, c1=1.0, c2=1.22, c3m=0.05, c3p=1.0,
                sigk=0.8, sigp=1.07),
}
GLS_PRESETS["k-psi"] = GLS_PRESETS["gen"]


def gls_preset(name="k-epsilon"):
    """GlsParams of a named GLS model (GLS_PRESETS)."""
    if name not in GLS_PRESETS:
        raise ValueError("GLS model must be one of %s" % sorted(GLS_PRESETS))
    P = GlsParams()
    for k, v in dict(_GLS_BASE, **GLS_PRESETS[name]).items():
        setattr(P, k, v)
    return P


def gls_defaults():
    """k-epsilon GLS (p=3, m=1.5, n=-1: utility/test.in:355-367) with the background and floor
    values of the GLS oracle."""
    return gls_preset("k-epsilon")


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


# -------------------------------------------------------------------------------------------
# column states and GLS runs
# -------------------------------------------------------------------------------------------
class Columns:
    """Water-column state of one basin for the closure: velocities at rho levels, buoyancy
    frequency, surface stress and the GLS turbulence fields, all on the current device."""

    def __init__(self, model, gls_model="k-epsilon"):
        self.m = model
        g = model.grid
        dt = model.tdtype
        dev = model.u.device
        N, J, I = g.N, g.J, g.I
        z = lambda *s: torch.zeros(*s, dtype=dt, device=dev)
        self.bvf = z(N + 1, J, I)
        self.sustr, self.svstr = z(J, I), z(J, I)
        self.gls_model = gls_model
        P = gls_preset(gls_model)
        self.P = P
        self.tke = torch.full((N + 1, J, I), P.Kmin, dtype=dt, device=dev)
        self.gls = torch.full((N + 1, J, I), P.Pmin, dtype=dt, device=dev)
        self.Akt, self.Akk, self.Akp = z(N + 1, J, I), z(N + 1, J, I), z(N + 1, J, I)
        self.Lscale = z(N + 1, J, I)
        self.Akt.fill_(P.Akt_bak)
        self.Akk.fill_(P.Akk_bak)
        self.Akp.fill_(P.Akp_bak)

    def stratify(self, zscale, dT=20.0):
        """N^2 of T = 4 + dT exp(z/zscale) with the linear EOS, from the model's z_w.  zscale is
        a number, or a (J, I) array of scales varying across the basin."""
        m = self.m
        if np.ndim(zscale) == 0:
            check(lib.sf_analytic_bvf(m.ctx.ptr, _p(m.z_w), dT, float(zscale), ALPHA, G,
                                      _p(self.bvf), stream_handle()), "sf_analytic_bvf")
            return
        zs = torch.as_tensor(np.asarray(zscale, np.float64), device=self.bvf.device)
        zw = m.z_w.double()
        self.bvf.copy_((G * ALPHA * (dT / zs) * torch.exp(zw / zs)).to(self.bvf.dtype))

    def gls_step(self, columns=None):
        m = self.m
        check(lib.sf_gls_corrector_cols(
            m.ctx.ptr, ctypes.byref(self.P), m.dt, _p(m.u), _p(m.v), _p(m.z_r), _p(m.Hz),
            _p(self.bvf), _p(self.sustr), _p(self.svstr), _p(self.tke), _p(self.gls), _p(m.AKv),
            _p(self.Akt), _p(self.Akk), _p(self.Akp), _p(self.Lscale), _p(columns),
            stream_handle()), "sf_gls_corrector_cols")

    def gls_step_list(self, lst, count):
        """Plain GLS on the columns lst[0 .. count) (device int32 list and count)."""
        m = self.m
        check(lib.sf_gls_corrector_list(
            m.ctx.ptr, ctypes.byref(self.P), m.dt, _p(m.u), _p(m.v), _p(m.z_r), _p(m.Hz),
            _p(self.bvf), _p(self.sustr), _p(self.svstr), _p(self.tke), _p(self.gls), _p(m.AKv),
            _p(self.Akt), _p(self.Akk), _p(self.Akp), _p(self.Lscale), _p(lst), _p(count),
            stream_handle()), "sf_gls_corrector_list")

    def features(self, X):
        m = self.m
        check(lib.sf_closure_features(m.ctx.ptr, _p(m.u), _p(m.v), _p(m.z_r), _p(self.bvf),
                                      _p(self.sustr), _p(self.svstr), _p(X), stream_handle()),
              "sf_closure_features")


def interior_columns(grid, device):
    idx = torch.arange(grid.s2, device=device)
    i, j = idx % grid.I, idx // grid.I
    return idx[(i != 0) & (i != grid.I - 1) & (j != 0) & (j != grid.J - 1)]


def wind_driven_state(model, cols, tau, angle, zscale, rng, current=True, pattern=False):
    """A wind-driven, stratified column state on the model's grid: surface stress tau (N/m2)
    at `angle` (times cos(pi y / Ly) if `pattern`, the basins' wind), a surface-intensified
    current decaying over an Ekman-like depth with a basin-scale gyre pattern and seeded
    small-scale noise (none if `current` is False: an ocean at rest under the wind), and the
    stratification of zscale."""
    if not model._started:
        model.start()
    g = model.grid
    dev = model.u.device
    dt = model.tdtype
    ustar2 = tau / RHO0
    if pattern:
        y = (torch.arange(g.J, device=dev, dtype=torch.float64) - 0.5) / max(g.J - 2, 1)
        shape = torch.cos(math.pi * y)[:, None].expand(g.J, g.I)
        cols.sustr.copy_((ustar2 * math.cos(angle) * shape).to(cols.sustr.dtype))
        cols.svstr.copy_((ustar2 * math.sin(angle) * shape).to(cols.svstr.dtype))
    else:
        cols.sustr.fill_(ustar2 * math.cos(angle))
        cols.svstr.fill_(ustar2 * math.sin(angle))
    if not current:
        model.u.zero_()
        model.v.zero_()
        cols.stratify(zscale)
        return
    ustar = math.sqrt(ustar2)
    d = max(5.0, 0.4 * ustar / 1e-4)                      # Ekman depth u*/f scale
    U0 = 40.0 * ustar2 / max(ustar, 1e-4) + 0.02          # surface drift ~ u*-proportional
    yy = torch.linspace(0, math.pi, g.J, device=dev, dtype=torch.float64)[:, None]
    xx = torch.linspace(0, math.pi, g.I, device=dev, dtype=torch.float64)[None, :]
    gyre_u = torch.cos(yy) * torch.sin(xx)
    gyre_v = -torch.sin(yy) * torch.cos(xx)
    z = model.z_r.double()
    prof = torch.exp(z / d)
    gen = torch.Generator(device=dev).manual_seed(int(rng.integers(1 << 31)))
    noise = lambda: 0.01 * U0 * torch.randn(z.shape, generator=gen, device=dev, dtype=torch.float64)
    ca, sa = math.cos(angle), math.sin(angle)
    u = U0 * prof * (ca + 0.5 * gyre_u) + noise()
    v = U0 * prof * (sa + 0.5 * gyre_v) + noise()
    model.u.zero_()
    model.v.zero_()
    model.u[:g.N] = u.to(dt)
    model.v[:g.N] = v.to(dt)
    cols.stratify(zscale)


def basin_forcing(model, cols, tau0=0.15, zscale=500.0):
    """The analytic basins' forcing for the closure: zonal wind stress tau0 cos(pi y / Ly)
    (N/m2, kinematic after division by rho0) and the stratification T = 4 + 20 exp(z/zscale)
    (N^2 from the model's z_w, so the depths are set first)."""
    if not model._started:
        model.start()
    g = model.grid
    J = g.J
    y = (torch.arange(J, device=model.u.device, dtype=torch.float64) - 0.5) / max(J - 2, 1)
    tau = tau0 * torch.cos(math.pi * y) / RHO0
    cols.sustr.copy_(tau[:, None].expand(J, g.I).to(cols.sustr.dtype))
    cols.svstr.zero_()
    cols.stratify(zscale)


def mixing_for(model, mode, net=None, tau0=0.15, zscale=500.0, gls_model=None):
    """A Closure for `model` ('gls' or 'mlp') under basin_forcing, installed as model.mixing;
    gls_model defaults to the network's (the model it was trained on), else k-epsilon."""
    c = Closure(model, mode, net, gls_model=gls_model)
    basin_forcing(model, c.cols, tau0, zscale)
    model.mixing = c
    return c


def generate(config="basin1", runs=4, spin=30, keep=4, every=5, seed=0, precision="fp32",
             tau_range=(0.0, 0.3), zscale_range=(200.0, 1000.0), rest_runs=0, pattern=False,
             spread=False, gls_model="k-epsilon"):
    """Training snapshots from plain GLS runs on `config`'s grid: each run draws a wind stress
    and a stratification scale, spins GLS up for `spin` steps at fixed forcing and then keeps
    `keep` snapshots `every` steps apart.  The last `rest_runs` of the runs have no current
    (an ocean at rest under the wind); with `pattern` the wind varies as cos(pi y / Ly), and
    with `spread` the stratification scale varies across xi over all of zscale_range.  Returns (X, T) on the device: feature rows and target
    rows (log10 Akv / Akt) of the rho-interior columns."""
    cfg = configs.CONFIGS[config]() if isinstance(config, str) else config
    g = cfg["grid"]
    if nfeat(g.N) > WIDTH:
        raise ValueError("the closure's rows hold at most 62 interior W levels")
    model = Model(g, cfg["boundary"], cfg["dt"], cfg["ndtfast"], precision=precision)
    model.start()
    dev = model.u.device
    cols_idx = interior_columns(g, dev)
    rng = np.random.default_rng(seed)
    nc = int(cols_idx.numel())
    # the rows go straight into preallocated tensors (no list of snapshots to concatenate:
    # tens of millions of rows are tens of GB)
    X = torch.empty((runs * keep * nc, WIDTH), device=dev)
    T = torch.empty((runs * keep * nc, WIDTH), device=dev)
    row = 0
    Xbuf = torch.zeros((g.s2, WIDTH), device=dev)
    for r in range(runs):
        cols = Columns(model, gls_model)
        tau = float(rng.uniform(*tau_range))
        angle = float(rng.uniform(0.0, 2.0 * math.pi))
        if spread:   # the stratification scale varies linearly across xi over the whole range
            lo, hi = zscale_range
            ramp = np.linspace(0.0, 1.0, g.I)[None, :] * np.ones((g.J, 1))
            if rng.random() < 0.5:
                ramp = 1.0 - ramp
            zscale = lo + (hi - lo) * ramp
        else:
            zscale = float(rng.uniform(*zscale_range))
        wind_driven_state(model, cols, tau, angle, zscale, rng, current=r < runs - rest_runs,
                          pattern=pattern)
        model.AKv.fill_(cols.P.Akv_bak)
        for it in range(spin + keep * every):
            cols.gls_step()
            if it >= spin and (it - spin) % every == every - 1:
                cols.features(Xbuf)
                X[row:row + nc] = Xbuf[cols_idx]
                T[row:row + nc] = targets(model.AKv, cols.Akt, g.N)[cols_idx]
                row += nc
    torch.cuda.synchronize()
    return X, T


def generate_roms(config="basin1", runs=6, hours=48.0, spin_hours=4.0, every=10, seed=0,
                  precision="fp32", tau_range=(0.0, 0.3), zscale_range=(200.0, 1000.0),
                  gls_model="k-epsilon", rdrag2=3e-3):
    """Training snapshots along ROMS-form model runs with plain GLS (the dynamics the closure
    replaces, including its transients): each run draws a peak wind stress from tau_range
    (zonal, cos(pi y / Ly) across the basin, either sign) and a stratification scale from
    zscale_range, starts from rest, and after `spin_hours` keeps a snapshot of the GLS
    columns (features, log10 Akv / Akt) every `every` steps until `hours`.  Returns (X, T) on
    the device for the rho-interior columns."""
    cfg = configs.CONFIGS[config]() if isinstance(config, str) else config
    g = cfg["grid"]
    if nfeat(g.N) > WIDTH:
        raise ValueError("the closure's rows hold at most 62 interior W levels")
    nd, _ = configs.roms_ndtfast(cfg)
    nsteps = int(round(hours * 3600.0 / cfg["dt"]))
    spin = int(round(spin_hours * 3600.0 / cfg["dt"]))
    keep = len(range(spin, nsteps, every))
    rng = np.random.default_rng(seed)
    X = T = None
    row = 0
    for r in range(runs):
        tau = float(rng.uniform(*tau_range)) * (1.0 if rng.random() < 0.5 else -1.0)
        zscale = float(rng.uniform(*zscale_range))
        m = Model(g, cfg["boundary"], cfg["dt"], nd, precision=precision, semantics="roms")
        c = mixing_for(m, "gls", None, tau0=tau, zscale=zscale, gls_model=gls_model)
        m.set_forcing(c.cols.sustr.double().cpu().numpy(), c.cols.svstr.double().cpu().numpy(),
                      rdrag2)
        dev = m.u.device
        if X is None:
            cols_idx = interior_columns(g, dev)
            nc = int(cols_idx.numel())
            X = torch.empty((runs * keep * nc, WIDTH), device=dev)
            T = torch.empty((runs * keep * nc, WIDTH), device=dev)
            Xbuf = torch.zeros((g.s2, WIDTH), device=dev)
        for k in range(nsteps):
            m.step(1)
            if k >= spin and (k - spin) % every == 0:
                c.cols.features(Xbuf)
                X[row:row + nc] = Xbuf[cols_idx]
                T[row:row + nc] = targets(m.AKv, c.cols.Akt, g.N)[cols_idx]
                row += nc
        del m, c
        torch.cuda.empty_cache()
    torch.cuda.synchronize()
    # a run that left the scheme's stability range leaves non-finite rows: drop them
    ok = torch.isfinite(X[:row]).all(1) & torch.isfinite(T[:row]).all(1)
    return X[:row][ok], T[:row][ok]


def targets(Akv, Akt, N):
    """Target rows (s2 x 128): log10 Akv at W levels 1..N-1 in [0, N-1), log10 Akt in
    [N-1, 2N-2)."""
    s2 = Akv[0].numel()
    nl = N - 1
    T = torch.zeros((s2, WIDTH), device=Akv.device)
    lv = torch.log10(Akv[1:N].reshape(nl, s2).float().clamp(1e-6, 1e-1))
    lt = torch.log10(Akt[1:N].reshape(nl, s2).float().clamp(1e-6, 1e-1))
    T[:, :nl] = lv.T
    T[:, nl:2 * nl] = lt.T
    return T


# -------------------------------------------------------------------------------------------
# the network and its training
# -------------------------------------------------------------------------------------------
class Network:
    """SF_MLP_LAYERS x 128 network (ReLU between layers by default, or GELU): FP32 master weights
    and Adam moments, BF16 copies for the tensor cores.  Inputs are normalised with the training set's per-feature mean and spread,
    which `inference_params()` folds into the first layer."""

    def __init__(self, N, seed=0, device="cuda", act="relu", gls_model="k-epsilon"):
        if nfeat(N) > WIDTH:
            raise ValueError("the closure's rows hold at most 62 interior W levels")
        if act not in MLP_ACT:
            raise ValueError("act must be one of %s" % sorted(MLP_ACT))
        self.N = int(N)
        self.act = act
        self.gls_model = gls_model   # the GLS model whose coefficients it learns
        gen = torch.Generator().manual_seed(seed)
        self.W = [(torch.randn(WIDTH, WIDTH, generator=gen) * math.sqrt(2.0 / WIDTH)).to(device)
                  for _ in range(LAYERS)]
        self.W[-1] *= 0.1
        self.b = [torch.zeros(WIDTH, device=device) for _ in range(LAYERS)]
        self.Wb = [w.to(torch.bfloat16) for w in self.W]
        self.mW = [torch.zeros_like(w) for w in self.W]
        self.vW = [torch.zeros_like(w) for w in self.W]
        self.mb = [torch.zeros_like(b) for b in self.b]
        self.vb = [torch.zeros_like(b) for b in self.b]
        self.mu = torch.zeros(WIDTH, device=device)
        self.isd = torch.ones(WIDTH, device=device)
        self.lo = torch.full((WIDTH,), -np.inf, device=device)
        self.hi = torch.full((WIDTH,), np.inf, device=device)
        self.step_count = 0
        self.err = torch.zeros(1, dtype=torch.int32, device=device)

    def params(self, W=None, b=None):
        P = MlpParams()
        W = W if W is not None else self.Wb
        b = b if b is not None else self.b
        for l in range(LAYERS):
            P.W[l] = W[l].data_ptr()
            P.b[l] = b[l].data_ptr()
        P.act = MLP_ACT[self.act]
        return P

    def inference_params(self):
        """(MlpParams, keep-alive tensors) for raw feature rows: the input normalisation
        folded into layer 0 (W0' = W0 diag(isd), b0' = b0 - W0' mu)."""
        W0 = self.W[0] * self.isd[None, :]
        b0 = self.b[0] - W0 @ self.mu
        Wb = [W0.to(torch.bfloat16)] + self.Wb[1:]
        b = [b0] + self.b[1:]
        return self.params(Wb, b), (Wb, b)

    def fit_normalisation(self, X):
        mu = X.mean(0)
        sd = X.std(0)
        self.mu = torch.where(sd > 1e-6, mu, torch.zeros_like(mu))
        self.isd = torch.where(sd > 1e-6, 1.0 / sd, torch.zeros_like(sd))
        self.mu[nfeat(self.N):] = 0.0
        self.isd[nfeat(self.N):] = 0.0
        lo, hi = X.min(0).values, X.max(0).values
        pad = 0.05 * (hi - lo) + 1e-3
        self.lo, self.hi = (lo - pad).contiguous(), (hi + pad).contiguous()

    def train(self, X, T, steps=2000, batch=2048, lr=2e-3, seed=0, log_every=0):
        """Adam on the MSE of the nout(N) trained outputs, minibatches drawn with a seeded
        permutation; every product on the tensor cores through sf_mlp_forward/backward."""
        dev = X.device
        n = X.shape[0]
        batch = min(batch, n - n % 16)
        Xn = (X - self.mu) * self.isd
        acts = torch.zeros((LAYERS - 1, batch, WIDTH), device=dev)
        pre = torch.zeros((LAYERS, batch, WIDTH), device=dev)
        Y = torch.zeros((batch, WIDTH), device=dev)
        dY = torch.zeros_like(Y)
        work = torch.zeros((2, batch, WIDTH), device=dev)
        dW = [torch.zeros(WIDTH, WIDTH, device=dev) for _ in range(LAYERS)]
        db = [torch.zeros(WIDTH, device=dev) for _ in range(LAYERS)]
        pdW = (ctypes.c_void_p * LAYERS)(*[t.data_ptr() for t in dW])
        pdb = (ctypes.c_void_p * LAYERS)(*[t.data_ptr() for t in db])
        loss = torch.zeros(1, device=dev)
        gen = torch.Generator(device=dev).manual_seed(seed)
        st = stream_handle()
        P = self.params()
        history = []
        perm = torch.randperm(n, generator=gen, device=dev)
        pos = 0
        for it in range(steps):
            if pos + batch > n:
                perm = torch.randperm(n, generator=gen, device=dev)
                pos = 0
            idx = perm[pos:pos + batch]
            pos += batch
            xb = Xn[idx].contiguous()
            tb = T[idx].contiguous()
            loss.zero_()
            check(lib.sf_mlp_forward(ctypes.byref(P), batch, _p(xb), _p(Y), _p(acts), _p(pre),
                                     _p(self.err), st), "sf_mlp_forward")
            check(lib.sf_mlp_mse(batch, nout(self.N), _p(Y), _p(tb), _p(dY), _p(loss), st),
                  "sf_mlp_mse")
            check(lib.sf_mlp_backward(ctypes.byref(P), batch, _p(xb), _p(acts), _p(pre), _p(dY),
                                      pdW, pdb, _p(work), _p(self.err), st), "sf_mlp_backward")
            self.step_count += 1
            for l in range(LAYERS):
                check(lib.sf_mlp_adam(WIDTH * WIDTH, _p(self.W[l]), _p(dW[l]), _p(self.mW[l]),
                                      _p(self.vW[l]), _p(self.Wb[l]), ctypes.c_float(lr),
                                      ctypes.c_float(0.9), ctypes.c_float(0.999), self.step_count,
                                      ctypes.c_float(1e-8), st), "sf_mlp_adam")
                check(lib.sf_mlp_adam(WIDTH, _p(self.b[l]), _p(db[l]), _p(self.mb[l]),
                                      _p(self.vb[l]), None, ctypes.c_float(lr), ctypes.c_float(0.9),
                                      ctypes.c_float(0.999), self.step_count, ctypes.c_float(1e-8),
                                      st), "sf_mlp_adam")
            if log_every and (it % log_every == 0 or it == steps - 1):
                history.append((it, float(loss.item())))
        if int(self.err.item()):
            raise RuntimeError("a tensor-core wait gave up during training")
        return history

    def save(self, path, **meta):
        """Master weights, normalisation and training range (NumPy .npz) plus `meta`."""
        np.savez(path, N=self.N, act=self.act, gls_model=self.gls_model,
                 W=np.stack([w.cpu().numpy() for w in self.W]),
                 b=np.stack([b.cpu().numpy() for b in self.b]), mu=self.mu.cpu().numpy(),
                 isd=self.isd.cpu().numpy(), lo=self.lo.cpu().numpy(), hi=self.hi.cpu().numpy(),
                 **{k: np.asarray(v) for k, v in meta.items()})

    @classmethod
    def load(cls, path, device="cuda"):
        d = np.load(path)
        # files without an activation entry hold GELU networks
        net = cls(int(d["N"]), device=device, act=str(d["act"]) if "act" in d else "gelu",
                  gls_model=str(d["gls_model"]) if "gls_model" in d else "k-epsilon")
        t = lambda a: torch.tensor(np.asarray(a, np.float32), device=device)
        net.W = [t(w) for w in d["W"]]
        net.b = [t(b) for b in d["b"]]
        net.Wb = [w.to(torch.bfloat16) for w in net.W]
        net.mu, net.isd, net.lo, net.hi = t(d["mu"]), t(d["isd"]), t(d["lo"]), t(d["hi"])
        return net

    def infer(self, X):
        """Outputs for raw feature rows X (n x 128) through the fused inference kernel."""
        P, keep = self.inference_params()
        Y = torch.empty_like(X)
        check(lib.sf_mlp_infer(ctypes.byref(P), X.shape[0], _p(X), _p(Y), _p(self.err),
                               stream_handle()), "sf_mlp_infer")
        return Y


def log_rms(Y, T, N):
    """RMS log10 error of Akv and Akt over the trained outputs (levels 1..N-1)."""
    nl = N - 1
    ev = (Y[:, :nl] - T[:, :nl]).double()
    et = (Y[:, nl:2 * nl] - T[:, nl:2 * nl]).double()
    return float(ev.pow(2).mean().sqrt()), float(et.pow(2).mean().sqrt())


# -------------------------------------------------------------------------------------------
# the closure inside the time step
# -------------------------------------------------------------------------------------------
class Closure:
    """Per-step vertical mixing for a Model: 'gls' runs plain GLS on every column; 'mlp' runs
    the network on every column and plain GLS on the columns outside its training range
    (fused: one sf_closure_step pass; otherwise features, range mask, sf_mlp_infer and
    sf_closure_apply as separate launches)."""

    def __init__(self, model, mode="mlp", net=None, fused=True, gls_model=None):
        if mode not in ("gls", "mlp"):
            raise ValueError("mode must be 'gls' or 'mlp'")
        if mode == "mlp" and net is None:
            raise ValueError("mode 'mlp' needs a trained Network")
        if mode == "mlp" and net.N != model.grid.N:
            raise ValueError("the network was trained for N=%d levels" % net.N)
        self.m, self.mode, self.net, self.fused = model, mode, net, fused
        # Model.step may run it beside the next step's first phases: it reads u, v, z_r, Hz,
        # bvf and the surface stress, and writes AKv and its own turbulence fields only
        self.overlappable = True
        if gls_model is None:
            gls_model = net.gls_model if net is not None else "k-epsilon"
        self.cols = Columns(model, gls_model)
        g = model.grid
        dev = model.u.device
        if mode == "mlp":
            if not fused:   # the unfused composition: features, mask, inference, update
                self.X = torch.zeros((g.s2, WIDTH), device=dev)
                self.Y = torch.zeros((g.s2, WIDTH), device=dev)
            self.mask = torch.zeros(g.s2, dtype=torch.uint8, device=dev)
            self.flist = torch.zeros(g.s2, dtype=torch.int32, device=dev)
            self.fcount = torch.zeros(1, dtype=torch.int32, device=dev)
            self.P, self._keep = net.inference_params()
            self.lo = net.lo.contiguous()
            self.hi = net.hi.contiguous()

    def __call__(self):
        m, c = self.m, self.cols
        if self.mode == "gls":
            c.gls_step()
            return
        st = stream_handle()
        if self.fused:
            check(lib.sf_closure_step(m.ctx.ptr, ctypes.byref(self.P), _p(m.u), _p(m.v),
                                      _p(m.z_r), _p(c.bvf), _p(c.sustr), _p(c.svstr),
                                      nfeat(m.grid.N), _p(self.lo), _p(self.hi), _p(self.mask),
                                      _p(self.flist), _p(self.fcount), _p(m.AKv), _p(c.Akt),
                                      _p(self.net.err), st), "sf_closure_step")
            c.gls_step_list(self.flist, self.fcount)   # plain GLS on the fallback columns
            return
        else:
            c.features(self.X)
            check(lib.sf_closure_range_mask(m.ctx.ptr, _p(self.X), nfeat(m.grid.N), _p(self.lo),
                                            _p(self.hi), _p(self.mask), st),
                  "sf_closure_range_mask")
            check(lib.sf_mlp_infer(ctypes.byref(self.P), m.grid.s2, _p(self.X), _p(self.Y),
                                   _p(self.net.err), st), "sf_mlp_infer")
            check(lib.sf_closure_apply(m.ctx.ptr, _p(self.Y), _p(self.mask), _p(m.AKv),
                                       _p(c.Akt), st), "sf_closure_apply")
        c.gls_step(self.mask)       # plain GLS on the fallback columns only
