"""The reference's own kernels (oracle/_ref, host-compiled by build_ref.py) driven in the
order of its Python orchestration -- the reference's CPU path of the time step.

TEST/BASELINE INFRASTRUCTURE: used by tests/ (to cross-check the oracle driver) and by
bench.py's reference arm and CPU-baseline leg, never by the product.

Launch geometry is the reference's (modules/mod_operators.py:40-41, utility/misc.py:10,17):
grsz*bksz threads for most kernels and grsz*GPUMUL*(bksz/GPUMUL) for the "x GPUMUL"
launches, which is the same count; boundary scatters use size/512+1 blocks of 512.
With omp > 1 the thread loop of each kernel is split over OpenMP threads (timing only: the
reference's own GPU launches are concurrent too, and the few kernels with races between
threads, e.g. rhs_kernels.cpp:86-91, then resolve them in no fixed order).
"""
import ctypes
import math
import os
import time

import numpy as np

from oracle import gzeros, P, D, Ii, G_GRAV

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(HERE, "_ref")
_vp, _d, _i, _u, _b, _l = (ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_uint,
                           ctypes.c_bool, ctypes.c_long)
SIGS = {
    "2d": {"initialize": [_u, _u, _u] + [_vp] * 4,
           "computeMomentumRHSPred": [_vp] * 5 + [_d, _d],
           "computeMomentumRHSCorr": [_vp] * 6 + [_d],
           "computeZetaRHS": [_vp] * 7 + [_b, _vp, _vp, _i, _vp],
           "computeZetaPred": [_d] + [_vp] * 4,
           "computeMomentumPred": [_d] + [_vp] * 9,
           "AdamsMoultonCorr3rd": [_d] + [_vp] * 4},
    "rhs": {"initialize": [_u, _u, _u] + [_vp] * 4,
            "addCoriolis": [_vp] * 6, "horizontalAdvection": [_vp] * 7,
            "verticalAdvection": [_vp] * 6},
    "step3d": {"initialize": [_u, _u, _u] + [_vp] * 4, "setVerticalVelEq": [_vp] * 3,
               "omega": [_vp] * 7, "set_depth": [_i] + [_vp] * 4 + [_d] + [_vp] * 5,
               "set_zeta": [_vp] * 3, "setLateralUVBCs": [_d] + [_vp] * 6,
               "set_maxflux": [_vp] * 5, "step3d_UV": [_vp] * 16 + [_i, _i, _d, _d, _d]},
    "bc": {"setBC": [_vp, _vp, _u, _d], "copyBC": [_vp, _vp, _vp, _u]},
}


def available(suffix=""):
    return all(os.path.exists(os.path.join(REF, "libsfref_%s%s.so" % (m, suffix))) for m in SIGS)


class RefKernels:
    """The reference's kernels from oracle/_ref; suffix "" is the pinned build (-O2, no
    contraction), "_native" the timed build (build_ref.build_native)."""

    def __init__(self, omp=1, suffix=""):
        self.omp = int(omp)
        self.libs = {}
        for mod, fns in SIGS.items():
            lib = ctypes.CDLL(os.path.join(REF, "libsfref_%s%s.so" % (mod, suffix)))
            for name, args in fns.items():
                f = getattr(lib, "sfref_" + name)
                f.argtypes = [_l, _i] + args
                f.restype = None
            self.libs[mod] = lib

    def __call__(self, mod, name, nthreads, *args):
        getattr(self.libs[mod], "sfref_" + name)(_l(nthreads), _i(self.omp), *args)


def _step2d_pair(K, grid, B, O, ct, nt, zetabc, velbc):
    """step2dPredictor (step2d.py:23-81) and step2dCorrector (:84-128) with the reference's
    kernels, on the current slot views of O; the predictor's leapfrog branch (iif >= 1)."""
    def pred():
        z0, z1, z2 = O.t("zeta", 0), O.t("zeta", 1), O.t("zeta", 2)
        Dt = ct.dtfast
        K("2d", "computeZetaRHS", nt, P(z1), P(grid.h), P(O.t("ubar", 1)), P(O.t("vbar", 1)),
          P(O.DU_avg1), P(O.DV_avg1), P(O.Zt_avg1), _b(True), P(ct.weight1), P(ct.weight2),
          Ii(ct.iif), P(O.t("rzeta", 1)))
        K("2d", "computeZetaPred", nt, D(Dt), P(z0), P(z1), P(z2), P(O.t("rzeta", 1)))
        zetabc(z2)
        K("2d", "computeMomentumRHSPred", nt, P(grid.h), P(O.t("rubar", 1)), P(O.t("rvbar", 1)),
          P(z0), P(z2), D(G_GRAV), D(2.0 / 5.0))
        K("2d", "computeMomentumPred", nt, D(Dt), P(O.t("ubar", 1)), P(O.t("ubar", 2)),
          P(O.t("vbar", 1)), P(O.t("vbar", 2)), P(O.t("rubar", 1)), P(O.t("rvbar", 1)),
          P(grid.h), P(z1), P(z2))
        velbc(O.t("ubar", 2), O.t("vbar", 2))

    def corr():
        z0, z1, z2 = O.t("zeta", 0), O.t("zeta", 1), O.t("zeta", 2)
        Dt = ct.dtfast
        K("2d", "computeZetaRHS", nt, P(z2), P(grid.h), P(O.t("ubar", 2)), P(O.t("vbar", 2)),
          P(O.DU_avg1), P(O.DV_avg1), P(O.Zt_avg1), _b(False), P(ct.weight1), P(ct.weight2),
          Ii(ct.iif), P(O.t("rzeta", 1)))
        K("2d", "AdamsMoultonCorr3rd", nt, D(Dt), P(z2), P(O.t("rzeta", 0)), P(O.t("rzeta", 1)),
          P(O.t("rzeta", 2)))
        zetabc(z2)
        K("2d", "computeMomentumRHSCorr", nt, P(grid.h), P(O.t("rubar", 2)), P(O.t("rvbar", 2)),
          P(z0), P(z1), P(z2), D(G_GRAV))
        K("2d", "AdamsMoultonCorr3rd", nt, D(Dt), P(O.t("ubar", 1)), P(O.t("vbar", 1)),
          P(O.t("rubar", 0)), P(O.t("rubar", 1)))
        velbc(O.t("ubar", 2), O.t("vbar", 2))

    return pred, corr


def _bc_fns(K, B, ct):
    bcn = lambda n: (n // 512 + 1) * 512

    def copy_bc(var, a1, a2, n):
        K("bc", "copyBC", bcn(n), P(var), P(a1), P(a2), ctypes.c_uint(n))

    def set_bc(var, a, val):
        K("bc", "setBC", bcn(a.size), P(var), P(a), ctypes.c_uint(a.size), D(val))

    def zetabc(z):
        copy_bc(z, B["zetaClosedOrGradientBCIdx1"], B["zetaClosedOrGradientBCIdx2"],
                B["zetaClosedOrGradientBCIdx1"].size)

    def velbc(ub, vb):
        set_bc(ub, B["ubarClosedBCIdx1"], 0.0)
        set_bc(vb, B["vbarClosedBCIdx1"], 0.0)
        set_bc(ub, B["ubarClampedBCIdx1"], .05 * math.sin(ct.time2D * 0.0002))
        copy_bc(ub, B["ubarGradientBCIdx1"], B["ubarGradientBCIdx2"], B["ubarGradientBCIdx1"].size)
        copy_bc(vb, B["vbarGradientBCIdx1"], B["ubarGradientBCIdx2"], B["vbarGradientBCIdx1"].size)

    return zetabc, velbc


def main2d(grid, B, O, ct, nsteps, omp=1):
    """nonlinear/main2d.py:9-88 with the reference's kernels: per 2D step next2DTimeStep,
    cycleTimes2D, step2dPredictor, step2dCorrector (no accumulator reset, vbar_t2 kept)."""
    K = RefKernels(omp)
    nt = (grid.s2 // 512 + 1) * 512
    args_init = (ctypes.c_uint(grid.N), ctypes.c_uint(grid.J), ctypes.c_uint(grid.I),
                 P(grid.on_u), P(grid.om_v), P(grid.pn), P(grid.pm))
    K("2d", "initialize", 1, *args_init)
    zetabc, velbc = _bc_fns(K, B, ct)
    pred, corr = _step2d_pair(K, grid, B, O, ct, nt, zetabc, velbc)
    for _ in range(nsteps):
        ct.next2d()
        O.cycle2d()
        pred()
        corr()


def main3d(grid, B, O, ct, nsteps, omp=1, lam=1.0, suffix="", kernels=None, step_marks=None):
    """nonlinear/main3d.py:25-326 with the reference's kernels (step2d.py, zetabc.py,
    barotropicVelocityBC.py, rhs.py orchestration restated), on oracle.Grid/Ocean/CompTimes.
    `step_marks`, if a list, receives time.perf_counter() at the end of every step."""
    K = kernels or RefKernels(omp, suffix)
    N, J, I = grid.N, grid.J, grid.I
    s2 = grid.s2
    nt = (s2 // 512 + 1) * 512          # grsz*bksz and grsz*GPUMUL*(bksz//GPUMUL)
    args_init = (ctypes.c_uint(N), ctypes.c_uint(J), ctypes.c_uint(I), P(grid.on_u), P(grid.om_v),
                 P(grid.pn), P(grid.pm))
    for mod in ("2d", "rhs", "step3d"):
        K(mod, "initialize", 1, *args_init)
    eq = [gzeros((N + 1, J, I)) for _ in range(3)]
    tmpU, tmpV = gzeros((N + 1) * J * I), gzeros((N + 1) * J * I)
    BC = B["zetaBC_bcIdxFieldIdx2"]
    K("step3d", "setVerticalVelEq", 1, P(eq[0]), P(eq[1]), P(eq[2]))

    def set_depth():
        K("step3d", "set_depth", nt, Ii(grid.Vtransform), P(O.Zt_avg1), P(grid.z_w), P(grid.z_r),
          P(grid.h), D(grid.hc), P(grid.Hz), P(grid.sc_r), P(grid.sc_w), P(grid.Cs_r), P(grid.Cs_w))

    zetabc, velbc = _bc_fns(K, B, ct)
    pred, corr = _step2d_pair(K, grid, B, O, ct, nt, zetabc, velbc)
    set_depth()
    for _ in range(nsteps):
        K("step3d", "set_maxflux", nt, P(O.t3("u")), P(O.t3("v")), P(O.Huon), P(O.Hvom), P(grid.Hz))
        K("step3d", "omega", nt, P(O.W), P(O.t3("u")), P(O.t3("v")), P(O.Huon), P(O.Hvom),
          P(grid.z_w), P(BC))
        K("step3d", "set_zeta", nt, P(O.t("zeta", 1)), P(O.t("zeta", 2)), P(O.Zt_avg1))
        ru, rv = O.t3("ru"), O.t3("rv")
        ru[:] = 0.0
        rv[:] = 0.0
        K("rhs", "addCoriolis", nt, P(grid.fomn), P(O.t3("u")), P(O.t3("v")), P(ru), P(rv), P(grid.Hz))
        K("rhs", "horizontalAdvection", nt, P(O.t3("u")), P(O.t3("v")), P(O.Huon), P(O.Hvom), P(ru),
          P(rv), P(BC))
        K("rhs", "verticalAdvection", nt, P(O.t3("u")), P(O.t3("v")), P(O.W), P(ru), P(rv), P(BC))
        ct.iif = 0
        for _ in range(ct.nfast + 1):
            if ct.iif == 0:
                O.Zt_avg1[:] = 0.0
                O.DU_avg1[:] = 0.0
                O.DV_avg1[:] = 0.0
            ct.next2d()
            O.cycle2d()
            pred()
            corr()
            O.t("vbar", 2)[:] = 0.0
        set_depth()
        tmpU[:] = O.t3("u")
        tmpV[:] = O.t3("v")
        K("step3d", "step3d_UV", nt, P(O.t3("u")), P(O.t3("v")), P(O.t3("ru")), P(O.t3("rv")),
          P(O.t("ubar", 1)), P(O.t("vbar", 1)), P(O.t("ubar", 2)), P(O.t("vbar", 2)), P(grid.Hz),
          P(O.AKv), P(grid.z_r), P(O.DU_avg1), P(O.DV_avg1), P(tmpU), P(tmpV), P(grid.h),
          Ii(ct.iic), Ii(ct.ntfirst), D(lam), D(1e-5), D(ct.dt))
        K("step3d", "setLateralUVBCs", nt, D(ct.time), P(O.t3("u")), P(O.t3("v")),
          P(B["uvelBC_bcIdxFieldIdx2"]), P(B["vvelBC_bcIdxFieldIdx2"]),
          P(B["uvelBC_bcIdxFieldType"]), P(B["vvelBC_bcIdxFieldType"]))
        K("step3d", "omega", nt, P(O.W), P(O.t3("u")), P(O.t3("v")), P(O.Huon), P(O.Hvom),
          P(grid.z_w), P(BC))
        ct.next3d()
        if step_marks is not None:
            step_marks.append(time.perf_counter())
