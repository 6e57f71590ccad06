"""Synthetic analytic basins of the benchmark and test configurations.

All inputs are analytic (no external data): depth from a tanh continental shelf across y plus
Gaussian seamounts, beta-plane Coriolis, S-coordinates with Vtransform 2 / Vstretching 4.

  basin0: config 0's 2D basin, Lm=128, Mm=64, dx=dy=5 km, flat h=4000 m, beta-plane f, dt=30 s
  basin1: Lm=512, Mm=256, N=32, dx=2 km, theta_s=5, theta_b=0.4, hc=100 m, one seamount,
          dt=240 s, ndtfast=30
  basin4: Lm=2048, Mm=1024, N=50, dx=1 km, same recipe with two seamounts, dt=120 s,
          ndtfast=40
  basin4q: Lm=1024, Mm=512, N=50, dx=2 km, basin4's recipe at a quarter of its area
"""
import numpy as np

from . import host
from .model import Grid

CLOSED = {k: "Clo Clo Clo Clo" for k in ("isFsur", "isUbar", "isVbar", "isUvel", "isVvel")}


def shelf_depth(Lm, Mm, dx, seamounts=(), shelf_frac=0.25, width_frac=0.1, hmin=50.0,
                hmax=4000.0, sm_height=2000.0, sm_radius=20.0e3):
    """Rho-point depth (Mm+2, Lm+2): hmin + (hmax-hmin)*tanh-shelf rising towards y=0, minus
    Gaussian seamounts of the given relative (x, y) positions, floored at hmin."""
    L, M = Lm + 1, Mm + 1
    jj, ii = np.meshgrid(np.arange(M + 1), np.arange(L + 1), indexing="ij")
    x, y = (ii - 0.5) * dx, (jj - 0.5) * dx
    Ly = Mm * dx
    Lx = Lm * dx
    prof = 0.5 * (1.0 + np.tanh((y - shelf_frac * Ly) / (width_frac * Ly)))
    h = hmin + (hmax - hmin) * prof
    for fx, fy in seamounts:
        h = h - sm_height * np.exp(-((x - fx * Lx) ** 2 + (y - fy * Ly) ** 2) / sm_radius ** 2)
    return np.maximum(h, hmin), x, y


def basin(Lm, Mm, N, dx, seamounts, dt, ndtfast, f0=1e-4, beta=2e-11, theta_s=5.0,
          theta_b=0.4, tcline=100.0, hflat=None):
    if hflat is None:
        h, x, y = shelf_depth(Lm, Mm, dx, seamounts)
    else:
        h, x, y = shelf_depth(Lm, Mm, dx)
        h[...] = hflat
    f = f0 + beta * (y - 0.5 * Mm * dx)
    grid = Grid.analytic(Lm, Mm, N, h, dx, dx, f, Vtransform=2, Vstretching=4, theta_s=theta_s,
                         theta_b=theta_b, tcline=tcline)
    grid.x, grid.y = x, y
    boundary = host.Boundary(grid.L, grid.M, CLOSED)
    return dict(grid=grid, boundary=boundary, dt=float(dt), ndtfast=int(ndtfast))


def basin0():
    """Config 0's grid: a flat 4000 m closed rectangle, Lm=128, Mm=64, dx=dy=5 km, beta-plane f,
    dt=30 s (one 2D step per call: ndtfast=1).  The 2D step uses no vertical levels; N=5 only
    satisfies the context's minimum."""
    return basin(128, 64, 5, 5.0e3, [], dt=30.0, ndtfast=1, hflat=4000.0)


# Lm, Mm, N, dx, seamounts (relative x, y), dt, ndtfast
PARAMS = {
    "basin1": (512, 256, 32, 2.0e3, [(0.5, 0.6)], 240.0, 30),
    "basin4": (2048, 1024, 50, 1.0e3, [(1.0 / 3.0, 0.6), (2.0 / 3.0, 0.6)], 120.0, 40),
    # a quarter of basin4 (dx = 2 km): the profiling case, with 3D fields of ~0.1 GB (FP32)
    # so that kernels stream from DRAM rather than L2
    "basin4q": (1024, 512, 50, 2.0e3, [(1.0 / 3.0, 0.6), (2.0 / 3.0, 0.6)], 120.0, 40),
}


def named(name, levels=None):
    """Basin `name` of PARAMS, optionally with another number of levels (the same horizontal
    grid, depth, dt and ndtfast: e.g. a profiling case for the 2D kernels)."""
    Lm, Mm, N, dx, mounts, dt, nd = PARAMS[name]
    return basin(Lm, Mm, levels or N, dx, mounts, dt=dt, ndtfast=nd)


def basin1():
    return named("basin1")


def basin4():
    return named("basin4")


def basin4q():
    return named("basin4q")


def small(Lm=256, Mm=128, N=32):
    return basin(Lm, Mm, N, 2.0e3, [(0.5, 0.6)], dt=240.0, ndtfast=30)


CONFIGS = {"basin0": basin0, "basin1": basin1, "basin4": basin4, "basin4q": basin4q, "small": small}


def roms_ndtfast(cfg, limit=0.65):
    """Barotropic substeps per baroclinic step for the ROMS-form step on `cfg`: its own
    ndtfast, raised where the fastest gravity wave (sqrt(g h_max)) would exceed c dtfast / dx
    = `limit` (the scheme is stable below 0.757 on a square grid: von Neumann analysis of the
    substep).  Returns (ndtfast, the configuration's own Courant number)."""
    g = cfg["grid"]
    nd = int(cfg["ndtfast"])
    courant = float(np.sqrt(10.0 * g.h.max()) * cfg["dt"] / nd * max(g.pm.max(), g.pn.max()))
    if courant > 0.7:
        nd = int(np.ceil(nd * courant / limit))
    return nd, courant
