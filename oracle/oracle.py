"""Oracle driver (TEST INFRASTRUCTURE): the reference's time step on the CPU in FP64.

``liboracle`` (oracle/sf_oracle.c) restates each reference kernel; this module restates the
reference's Python orchestration around them:

* nonlinear/step2d.py:23-128      step2dPredictor / step2dCorrector
* nonlinear/zetabc.py:5-12,
  nonlinear/barotropicVelocityBC.py:7-31   boundary scatters
* nonlinear/rhs.py:16-93          rhs3d
* nonlinear/main3d.py:25-326      the baroclinic step loop
* modules/mod_ocean.py:120-154    time-slot rotation (three-slot parents, views rotated)

Every array lives inside a zero-guarded parent (``gzeros``), so the reference kernels'
out-of-bounds reads at the boundary ring read zeros, as in tests/golden/make_golden.py.

Only tests/, __graft_entry__.smoke() and bench.py (CPU-baseline leg) may import this module.
"""
import ctypes
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
GUARD = 1 << 16


def build(verbose=False):
    src = os.path.join(HERE, "sf_oracle.c")
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(src):
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    cmd = ["gcc", "-std=c99", "-O2", "-fPIC", "-shared", "-ffp-contract=off", src, "-o", LIB, "-lm"]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build())
    return _lib


def gzeros(shape, dtype=np.float64):
    """Zero array inside a zero guard of GUARD elements on each side."""
    shape = tuple(shape) if isinstance(shape, (tuple, list)) else (int(shape),)
    n = int(np.prod(shape))
    parent = np.zeros(n + 2 * GUARD, dtype=dtype)
    return parent[GUARD:GUARD + n].reshape(shape)


def gcopy(a, dtype=None):
    a = np.asarray(a)
    out = gzeros(a.shape, dtype or a.dtype)
    out[...] = a
    return out


class OrcGrid(ctypes.Structure):
    _fields_ = [("I", ctypes.c_int), ("J", ctypes.c_int), ("N", ctypes.c_int),
                ("on_u", ctypes.c_void_p), ("om_v", ctypes.c_void_p),
                ("pn", ctypes.c_void_p), ("pm", ctypes.c_void_p)]


def P(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else ctypes.c_void_p(0)


def D(x):
    return ctypes.c_double(float(x))


def Ii(x):
    return ctypes.c_int(int(x))


def Li(x):
    return ctypes.c_long(int(x))


def reference_threads_2x(s2, block=512):
    """Thread count of the reference's (grsz*GPUMUL, bksz//GPUMUL) launches
    (modules/mod_operators.py:40-41, utility/misc.py:10,17)."""
    return (s2 // block + 1) * block


class Grid:
    """Grid arrays for the oracle: metrics (guarded FP64) and vertical coordinates."""

    def __init__(self, L, M, N, h, pm, pn, on_u, om_v, fomn, sc_r, sc_w, Cs_r, Cs_w, hc, Vtransform):
        self.L, self.M, self.N = int(L), int(M), int(N)
        self.I, self.J = self.L + 1, self.M + 1
        self.s2 = self.I * self.J
        g = lambda a: gcopy(np.asarray(a, np.float64).reshape(self.J, self.I))
        self.h, self.pm, self.pn, self.on_u, self.om_v, self.fomn = map(g, (h, pm, pn, on_u, om_v, fomn))
        self.sc_r, self.sc_w, self.Cs_r, self.Cs_w = (gcopy(np.asarray(a, np.float64)) for a in (sc_r, sc_w, Cs_r, Cs_w))
        self.hc, self.Vtransform = float(hc), int(Vtransform)
        self.z_w = gzeros((self.N + 1, self.J, self.I))
        self.z_r = gzeros((self.N, self.J, self.I))
        self.Hz = gzeros((self.N, self.J, self.I))
        self.c = OrcGrid(self.I, self.J, self.N, self.on_u.ctypes.data, self.om_v.ctypes.data,
                         self.pn.ctypes.data, self.pm.ctypes.data)

    @property
    def ref(self):
        return ctypes.c_void_p(ctypes.addressof(self.c))


class Boundary:
    """Boundary index arrays as built by modules/mod_boundary.py:237-297 (passed in)."""

    def __init__(self, arrays):
        self.a = {k: gcopy(np.asarray(v, np.int32)) for k, v in arrays.items()}

    def __getitem__(self, k):
        return self.a[k]


class Ocean:
    """Three-slot 2D/3D state of modules/mod_ocean.py:14-116 with its rotation."""

    NAMES2 = ("zeta", "ubar", "vbar", "rzeta", "rubar", "rvbar")
    NAMES3 = ("u", "v", "ru", "rv")

    def __init__(self, grid, init=None):
        J, I, N = grid.J, grid.I, grid.N
        for n in self.NAMES2:
            setattr(self, n, gzeros((3, J, I)))
        for n in self.NAMES3:
            setattr(self, n, gzeros((3, N + 1, J, I)))
        for n in ("W", "Huon", "Hvom"):
            setattr(self, n, gzeros((N + 1, J, I)))
        for n in ("Zt_avg1", "DU_avg1", "DV_avg1"):
            setattr(self, n, gzeros(J * I))
        self.AKv = gcopy(np.full((N + 1, J, I), 0.001))   # modules/mod_ocean.py:91
        self.slots = {n: [0, 1, 2] for n in self.NAMES2}
        if init is not None:
            for n, v in init.items():
                getattr(self, n)[...] = np.asarray(v).reshape(getattr(self, n).shape)

    def t(self, name, k):
        return getattr(self, name)[self.slots[name][k]].reshape(-1)

    def t3(self, name):     # 3D fields: only slot 2 is used (cycleTimes3D is never called)
        return getattr(self, name)[2].reshape(-1)

    def cycle2d(self):      # modules/mod_ocean.py:120-154
        for n in self.NAMES2:
            s = self.slots[n]
            self.slots[n] = [s[1], s[2], s[0]]


class CompTimes:
    """Counters of modules/mod_comptimes.py:7-108 used on the step path."""

    def __init__(self, dt, ndtfast, nfast, weight1, weight2):
        self.dt, self.ndtfast = float(dt), int(ndtfast)
        self.dtfast = self.dt / self.ndtfast
        self.nfast = int(nfast)
        self.weight1 = gcopy(np.asarray(weight1, np.float64))
        self.weight2 = gcopy(np.asarray(weight2, np.float64))
        self.iic = 0
        self.iif = 0
        self.time = 0.0
        self.time2D = 0.0
        self.ntfirst = 0

    def next2d(self):
        self.iif += 1
        self.time2D += self.dtfast

    def next3d(self):
        self.iic += 1
        self.time += self.dt
        self.time2D = self.time


G_GRAV = 10.0   # modules/mod_constants.py:26


# --------------------------------------------------------------------------------------
# Reference Python routines restated over the oracle kernels
# --------------------------------------------------------------------------------------
def zetabc(grid, B, zeta):          # nonlinear/zetabc.py:5-12
    a1, a2 = B["zetaClosedOrGradientBCIdx1"], B["zetaClosedOrGradientBCIdx2"]
    lib().orc_copy_bc(P(zeta), P(a1), P(a2), Li(a1.size))


def barotropic_velocity_bc(grid, B, ubar, vbar, time2D):   # nonlinear/barotropicVelocityBC.py:7-31
    L = lib()
    L.orc_set_bc(P(ubar), P(B["ubarClosedBCIdx1"]), Li(B["ubarClosedBCIdx1"].size), D(0.0))
    L.orc_set_bc(P(vbar), P(B["vbarClosedBCIdx1"]), Li(B["vbarClosedBCIdx1"].size), D(0.0))
    val = .05 * math.sin(time2D * 0.0002)
    L.orc_set_bc(P(ubar), P(B["ubarClampedBCIdx1"]), Li(B["ubarClampedBCIdx1"].size), D(val))
    L.orc_copy_bc(P(ubar), P(B["ubarGradientBCIdx1"]), P(B["ubarGradientBCIdx2"]),
                  Li(B["ubarGradientBCIdx1"].size))
    n = B["vbarGradientBCIdx1"].size
    if n > B["ubarGradientBCIdx2"].size:
        raise ValueError("vbar gradient boundary list longer than the ubar one the reference copies from")
    L.orc_copy_bc(P(vbar), P(B["vbarGradientBCIdx1"]), P(B["ubarGradientBCIdx2"]), Li(n))


def step2d_predictor(grid, B, O, ct):       # nonlinear/step2d.py:23-81
    L = lib()
    z2, z1, z0 = O.t("zeta", 2), O.t("zeta", 1), O.t("zeta", 0)
    Dt = ct.dtfast
    L.orc_zeta_rhs(grid.ref, P(z1), P(grid.h), P(O.t("ubar", 1)), P(O.t("vbar", 1)), P(O.DU_avg1),
                   P(O.DV_avg1), P(O.Zt_avg1), Ii(1), P(ct.weight1), Ii(ct.iif), P(O.t("rzeta", 1)))
    if ct.iif == 0:     # compTimes.isFirst2DStep(); never true inside main3d
        z2[:] = z1 + Dt * O.t("rzeta", 1)
        w = 0.5
    else:
        L.orc_zeta_pred(grid.ref, D(Dt), P(z0), P(z2), P(O.t("rzeta", 1)))
        w = 2.0 / 5.0
    zetabc(grid, B, z2)
    L.orc_momentum_rhs(grid.ref, P(grid.h), P(O.t("rubar", 1)), P(O.t("rvbar", 1)), P(z2), P(z0),
                       D(G_GRAV), D(w))
    L.orc_momentum_pred(grid.ref, D(Dt), P(O.t("ubar", 1)), P(O.t("ubar", 2)), P(O.t("vbar", 1)),
                        P(O.t("vbar", 2)), P(O.t("rubar", 1)), P(O.t("rvbar", 1)), P(grid.h),
                        P(z1), P(z2))
    barotropic_velocity_bc(grid, B, O.t("ubar", 2), O.t("vbar", 2), ct.time2D)


def step2d_corrector(grid, B, O, ct):       # nonlinear/step2d.py:84-128
    L = lib()
    z2 = O.t("zeta", 2)
    Dt = ct.dtfast
    L.orc_zeta_rhs(grid.ref, P(z2), P(grid.h), P(O.t("ubar", 2)), P(O.t("vbar", 2)), P(O.DU_avg1),
                   P(O.DV_avg1), P(O.Zt_avg1), Ii(0), P(ct.weight1), Ii(ct.iif), P(O.t("rzeta", 1)))
    L.orc_am3(grid.ref, D(Dt), P(z2), P(O.t("rzeta", 0)), P(O.t("rzeta", 1)), P(O.t("rzeta", 2)))
    zetabc(grid, B, z2)
    L.orc_momentum_rhs(grid.ref, P(grid.h), P(O.t("rubar", 2)), P(O.t("rvbar", 2)), P(z2),
                       P(O.t("zeta", 1)), D(G_GRAV), D(2.0 / 5.0))
    # AdamsMoultonCorr3rd2 is bound to AdamsMoultonCorr3rd (modules/mod_operators.py:146):
    L.orc_am3(grid.ref, D(Dt), P(O.t("ubar", 1)), P(O.t("vbar", 1)), P(O.t("rubar", 0)),
              P(O.t("rubar", 1)))
    barotropic_velocity_bc(grid, B, O.t("ubar", 2), O.t("vbar", 2), ct.time2D)


def main2d(grid, B, O, ct, nsteps):         # nonlinear/main2d.py:9-88
    """Per 2D step: next2DTimeStep, cycleTimes2D, step2dPredictor, step2dCorrector."""
    for _ in range(nsteps):
        ct.next2d()
        O.cycle2d()
        step2d_predictor(grid, B, O, ct)
        step2d_corrector(grid, B, O, ct)


def rhs3d(grid, B, O):                      # nonlinear/rhs.py:16-93
    L = lib()
    BC = B["zetaBC_bcIdxFieldIdx2"]
    ru, rv = O.t3("ru"), O.t3("rv")
    ru[:] = 0.0
    rv[:] = 0.0
    L.orc_add_coriolis(grid.ref, P(grid.fomn), P(O.t3("u")), P(O.t3("v")), P(ru), P(rv), P(grid.Hz))
    L.orc_horizontal_advection(grid.ref, P(O.t3("u")), P(O.t3("v")), P(O.Huon), P(O.Hvom), P(ru),
                               P(rv), Li(reference_threads_2x(grid.s2)))
    L.orc_vertical_advection(grid.ref, P(O.t3("u")), P(O.t3("v")), P(O.W), P(ru), P(rv), P(BC))


def set_depth(grid, O):
    lib().orc_set_depth(grid.ref, Ii(grid.Vtransform), P(O.Zt_avg1), P(grid.z_w), P(grid.z_r),
                        P(grid.h), D(grid.hc), P(grid.Hz), P(grid.sc_r), P(grid.sc_w),
                        P(grid.Cs_r), P(grid.Cs_w))


def main3d(grid, B, O, ct, nsteps, lam=1.0):
    """nonlinear/main3d.py:25-326 for `nsteps` baroclinic steps."""
    L = lib()
    N, J, I = grid.N, grid.J, grid.I
    eq = [gzeros((N + 1, J, I)) for _ in range(3)]
    tmpU, tmpV = gzeros((N + 1) * J * I), gzeros((N + 1) * J * I)
    BC = B["zetaBC_bcIdxFieldIdx2"]
    set_depth(grid, O)
    for _ in range(nsteps):
        L.orc_set_maxflux(grid.ref, P(O.t3("u")), P(O.t3("v")), P(O.Huon), P(O.Hvom), P(grid.Hz))
        L.orc_omega(grid.ref, P(O.W), P(O.Huon), P(O.Hvom), P(grid.z_w), P(BC))
        L.orc_set_zeta(grid.ref, P(O.t("zeta", 1)), P(O.t("zeta", 2)), P(O.Zt_avg1))
        rhs3d(grid, B, O)
        ct.iif = 0
        for _ in range(ct.nfast + 1):
            if ct.iif == 0:
                O.Zt_avg1[:] = 0.0
                O.DU_avg1[:] = 0.0
                O.DV_avg1[:] = 0.0
            ct.next2d()
            O.cycle2d()
            step2d_predictor(grid, B, O, ct)
            step2d_corrector(grid, B, O, ct)
            O.t("vbar", 2)[:] = 0.0
        set_depth(grid, O)
        tmpU[:] = O.t3("u")
        tmpV[:] = O.t3("v")
        L.orc_step3d_uv(grid.ref, P(O.t3("u")), P(O.t3("v")), P(O.t3("ru")), P(O.t3("rv")),
                        P(O.t("ubar", 1)), P(O.t("vbar", 1)), P(O.t("ubar", 2)), P(O.t("vbar", 2)),
                        P(grid.Hz), P(O.AKv), P(grid.z_r), P(O.DU_avg1), P(O.DV_avg1), P(tmpU),
                        P(tmpV), Ii(ct.iic), Ii(ct.ntfirst), D(lam), D(ct.dt), P(eq[0]), P(eq[1]),
                        P(eq[2]))
        L.orc_lateral_uv_bc(grid.ref, D(ct.time), P(O.t3("u")), P(O.t3("v")),
                            P(B["vvelBC_bcIdxFieldIdx2"]), P(B["uvelBC_bcIdxFieldType"]),
                            P(B["vvelBC_bcIdxFieldType"]))
        L.orc_omega(grid.ref, P(O.W), P(O.Huon), P(O.Hvom), P(grid.z_w), P(BC))
        ct.next3d()


def _argtypes():
    L = lib()
    vp, d, i, lg = ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_long
    sig = {
        "orc_zeta_rhs": [vp] * 8 + [i, vp, i, vp],
        "orc_zeta_pred": [vp, d, vp, vp, vp],
        "orc_momentum_rhs": [vp] * 6 + [d, d],
        "orc_momentum_pred": [vp, d] + [vp] * 9,
        "orc_am3": [vp, d, vp, vp, vp, vp],
        "orc_am3_momentum": [vp, d] + [vp] * 11,
        "orc_set_bc": [vp, vp, lg, d],
        "orc_copy_bc": [vp, vp, vp, lg],
        "orc_add_coriolis": [vp] * 7,
        "orc_horizontal_advection": [vp] * 7 + [lg],
        "orc_vertical_advection": [vp] * 7,
        "orc_set_maxflux": [vp] * 6,
        "orc_omega": [vp] * 6,
        "orc_set_zeta": [vp] * 4,
        "orc_set_depth": [vp, i] + [vp] * 4 + [d] + [vp] * 5,
        "orc_lateral_uv_bc": [vp, d] + [vp] * 5,
        "orc_step3d_uv": [vp] * 16 + [i, i, d, d] + [vp] * 3,
    }
    for n, a in sig.items():
        f = getattr(L, n)
        f.argtypes = a
        f.restype = None


_argtypes()
