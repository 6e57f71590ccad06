"""Ensembles of independent basins of uneven size, stepped together (config 2).

All members' fields live in shared pools (member after member, from sf_ctx_member_layout);
each time-step launch covers every member, each block finding its member from a block map
(sf_ctx_create_ensemble), so a step costs the same number of launches as one basin, and the
barotropic loop of all members replays as one CUDA graph.  The step itself is Model.step, in
either of its semantics: the reference's main3d per member, or the ROMS form (wind, drag,
Coriolis, closed walls: make(..., semantics="roms") and roms_forcing), which, unlike the
reference's step on the members' non-square grids, stays finite and so gives each member's
FP32 error against FP64.

    members = ensemble_members(seed=0, n=256)        # config 2: sizes, depths, bumps
    ens = make(members, precision="fp32")            # an Ensemble with the bumps loaded
    ens.step(10)
    zeta_m = ens.member("zeta", m)                   # a member's view in the reference shape
"""
import ctypes

import numpy as np
import torch

from . import configs
from ._lib import GridDesc, check, lib
from .model import DTYPES, Model, grid_desc


class EnsembleContext:
    """An sf_ctx over several grids (members) and its pool layout."""

    def __init__(self, members, precision="fp32"):
        if precision not in DTYPES:
            raise ValueError("precision must be 'fp64' or 'fp32'")
        self.precision = precision
        self.grids = [g for g, _ in members]
        self.n = len(members)
        self._keep = [{} for _ in members]
        descs = (GridDesc * self.n)()
        for m, (g, b) in enumerate(members):
            descs[m] = grid_desc(g, b, precision, self._keep[m])
        ptr = ctypes.c_void_p()
        check(lib.sf_ctx_create_ensemble(descs, self.n, ctypes.byref(ptr)),
              "sf_ctx_create_ensemble")
        self.ptr = ptr
        off2, off3, offN = ((ctypes.c_long * self.n)() for _ in range(3))
        tot = (ctypes.c_long * 3)()
        check(lib.sf_ctx_member_layout(ptr, off2, off3, offN, tot), "sf_ctx_member_layout")
        self.off2, self.off3, self.offN = list(off2), list(off3), list(offN)
        self.tot2, self.tot3, self.totN = tot[0], tot[1], tot[2]

    def close(self):
        if getattr(self, "ptr", None):
            lib.sf_ctx_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _Pool:
    """What Model.step needs of `grid` for pooled fields: the 2D pool's row length."""

    def __init__(self, s2):
        self.s2 = s2


class Ensemble(Model):
    """Model over an ensemble context: the same step, on pooled fields."""

    def __init__(self, members, dt, ndtfast, precision="fp32", lam=1.0, device="cuda",
                 semantics="reference"):
        """semantics: "reference" (the reference's main3d per member) or "roms" (the ROMS-form
        step per member: wind stress, quadratic bottom drag, Coriolis, closed walls; forcing
        through set_forcing on the pooled stress arrays or roms_forcing)."""
        from . import host
        if semantics not in ("reference", "roms"):
            raise ValueError("semantics must be 'reference' or 'roms'")
        self.ctx = EnsembleContext(members, precision)
        c = self.ctx
        self.members_grids = c.grids
        self.grid = _Pool(c.tot2)
        self.precision = precision
        self.tdtype = DTYPES[precision][1]
        self.dt, self.ndtfast = float(dt), int(ndtfast)
        self.dtfast = self.dt / self.ndtfast
        self.nfast, self.weight1, self.weight2 = host.set_weights(self.ndtfast)
        self._w1 = np.ascontiguousarray(self.weight1)
        self.lam = float(lam)
        self.iic, self.ntfirst = 0, 0
        self.time, self.time2D = 0.0, 0.0
        z = lambda *s, dt=None: torch.zeros(*s, dtype=dt or self.tdtype, device=device)
        for n in self.NAMES2:
            setattr(self, n, z(3, c.tot2))
        for n in self.NAMES3:
            setattr(self, n, z(c.tot3))
        self.AKv.fill_(0.001)                     # modules/mod_ocean.py:91
        for n in ("Zt_avg1", "DU_avg1", "DV_avg1"):
            setattr(self, n, z(c.tot2, dt=torch.float64))
        self.z_w = z(c.tot3)
        self.z_r = z(c.totN)
        self.Hz = z(c.totN)
        self.slots = [0, 1, 2]
        self._started = False
        self.mixing = None
        self.check_every = 0          # sf_check_state covers single grids only
        self.semantics = semantics
        if semantics == "roms":
            # as Model: ROMS-indexed averaging weights, the second fast-time averages, the
            # stresses and the Adams-Bashforth right-hand sides, on the pools
            self.W1, self.W2 = host.roms_weights(self.nfast, self.weight1)
            self.DU_avg2 = z(c.tot2, dt=torch.float64)
            self.DV_avg2 = z(c.tot2, dt=torch.float64)
            self.sustr = z(c.tot2)
            self.svstr = z(c.tot2)
            self.rdrag2 = 0.0
            self._ru3 = [self.ru, z(c.tot3), z(c.tot3)]
            self._rv3 = [self.rv, z(c.tot3), z(c.tot3)]
        self.cells = sum((g.L - 1) * (g.M - 1) * g.N for g in c.grids)

    KIND = {"zeta": 2, "ubar": 2, "vbar": 2, "rzeta": 2, "rubar": 2, "rvbar": 2, "Zt_avg1": 2,
            "DU_avg1": 2, "DV_avg1": 2, "u": 3, "v": 3, "ru": 3, "rv": 3, "W": 3, "Huon": 3,
            "Hvom": 3, "AKv": 3, "z_w": 3, "z_r": "N", "Hz": "N"}

    def member(self, name, m, slot=2):
        """Member m's part of a field as a view in the reference's shape ((M+1, L+1) for 2D
        fields, time slot `slot` of the three-slot ones; (levels, M+1, L+1) for 3D)."""
        g = self.members_grids[m]
        c = self.ctx
        kind = self.KIND[name]
        t = getattr(self, name)
        if name in self.NAMES2:
            t = t[self.slots[slot]]
        if kind == 2:
            return t[c.off2[m]:c.off2[m] + g.s2].view(g.J, g.I)
        lv = g.N + 1 if kind == 3 else g.N
        off = c.off3[m] if kind == 3 else c.offN[m]
        return t[off:off + lv * g.s2].view(lv, g.J, g.I)


def ensemble_members(seed=0, n=256, lm=(64, 512), mm=(32, 256), levels=(16, 32), dx=2.0e3,
                     amp=0.1, radius=50.0e3):
    """Config 2's members, drawn from numpy.random.default_rng(seed): Lm ~ U[64, 512],
    Mm ~ U[32, 256], N from {16, 32}, each with basin1's recipe (tanh shelf across y and a
    Gaussian seamount, both scaled to the member's size; dx, dt, theta_s, theta_b, hc as basin1)
    and an initial Gaussian surface bump of amplitude U[-amp, amp] and the given radius at a
    random position.  Returns [(grid, boundary, zeta0)]."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        Lm = int(rng.integers(lm[0], lm[1] + 1))
        Mm = int(rng.integers(mm[0], mm[1] + 1))
        N = int(rng.choice(levels))
        cfg = configs.basin(Lm, Mm, N, dx, [(0.5, 0.6)], dt=240.0, ndtfast=30)
        g = cfg["grid"]
        a = float(rng.uniform(-amp, amp))
        x0 = float(rng.uniform(0, Lm * dx))
        y0 = float(rng.uniform(0, Mm * dx))
        zeta0 = a * np.exp(-((g.x - x0) ** 2 + (g.y - y0) ** 2) / radius ** 2)
        out.append((g, cfg["boundary"], zeta0))
    return out


def roms_forcing(ens, tau0=0.1, rdrag2=3e-3):
    """Config 1's forcing on every member of a ROMS-form ensemble: zonal wind stress tau0
    cos(pi y / Ly) N/m2 over each member's own width (kinematic: divided by rho0 = 1025
    kg/m3, y the rho rows' distance from the south wall), quadratic bottom drag rdrag2."""
    c = ens.ctx
    tau = np.zeros(c.tot2)
    for m, g in enumerate(ens.members_grids):
        y = (np.arange(g.J, dtype=np.float64) - 0.5) / max(g.J - 2, 1)
        t = tau0 * np.cos(np.pi * y) / 1025.0
        tau[c.off2[m]:c.off2[m] + g.s2] = np.repeat(t, g.I)
    ens.set_forcing(tau, np.zeros(c.tot2), rdrag2)


def make(members, precision="fp32", dt=240.0, ndtfast=30, semantics="reference"):
    """An Ensemble of `members` (from ensemble_members) with their initial bumps in Zt_avg1
    (main3d.py:62 derives the depths from it) and zeta."""
    ens = Ensemble([(g, b) for g, b, _ in members], dt, ndtfast, precision, semantics=semantics)
    for m, (g, _, z0) in enumerate(members):
        zt = torch.from_numpy(np.ascontiguousarray(z0, np.float64).ravel()).to(ens.Zt_avg1.device)
        c = ens.ctx
        ens.Zt_avg1[c.off2[m]:c.off2[m] + g.s2] = zt
        for k in range(3):
            ens.zeta[k][c.off2[m]:c.off2[m] + g.s2] = zt.to(ens.tdtype)
    return ens
