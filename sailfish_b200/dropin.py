"""Drop-in replacements for the reference's Python entry points of the time step.

Same names, same arguments, same in-place effect on the same arrays as

    step2dPredictor(compTimes, GRID, OCEAN, BOUNDARY)      nonlinear/step2d.py:23-81
    step2dCorrector(compTimes, GRID, OCEAN, BOUNDARY)      nonlinear/step2d.py:84-128
    zetabc(zeta, compTimes, BOUNDARY)                      nonlinear/zetabc.py:5-12
    barotropicVelocityBC(ubar, vbar, compTimes, BOUNDARY)  nonlinear/barotropicVelocityBC.py:7-31
    rhs3d(GRID, OCEAN, BOUNDARY)                           nonlinear/rhs.py:16-93

and RawKernel-style callables with the reference's ``kernel(grid, block, args)`` convention
(cp.RawModule.get_function, modules/mod_operators.py:175-185); the launch geometry is
ignored, each call launches its own:

    set_maxflux((u, v, Huon, Hvom, Hz))                    step3D_uv.kernels.cpp:372-405
    omega((W, u, v, Huon, Hvom, z_w, BC))                  step3D_uv.kernels.cpp:62-165
    set_zeta((zeta_t1, zeta_t2, Zt_avg1))                  step3D_uv.kernels.cpp:294-310
    set_depth((Vtransform, Zt_avg1, z_w, z_r, h, hc, Hz, sc_r, sc_w, Cs_r, Cs_w))   :225-291
    step3d_UV((u, v, ru, rv, ubar_t1, vbar_t1, ubar_t2, vbar_t2, Hz, AKv, z_r, DU_avg1,
               DV_avg1, tmpU, tmpV, h, iic, ntfirst, lambda, AK, dt))               :646-707
    setLateralUVBCs((time, u, v, uIdx, vIdx, uType, vType))                          :314-368

plus ``gls_predictor_step(compTimes, GRID, OCEAN, MIXING)`` and
``gls_corrector_step(compTimes, GRID, OCEAN, MIXING, FORCES)``, which the reference names
(nonlinear/gls_predictor_step.py, nonlinear/gls_corrector_step.py) but never made runnable.

Arrays are any CUDA array exposing ``__cuda_array_interface__`` (CuPy arrays as the
reference allocates them, torch CUDA tensors, ...), C-contiguous, in the reference's flat
layout.  ``initModule(GRID, BOUNDARY)`` replaces mod_operators.initModule
(modules/mod_operators.py:31-45): like the reference's device globals, it holds one grid per
process.  Errors raise SailfishError (the reference has no error returns: CuPy raises on
launch failure and msgError exits).  Calls are asynchronous on `stream` (default: the legacy
default stream, which is CuPy's and torch's default).
"""
import ctypes

import numpy as np

from . import host
from ._lib import GlsParams, SailfishError, State2D, check, lib
from .model import Context, Grid

_ctx = None
_prec = None
stream = ctypes.c_void_p(0)


def _host(a):
    """Host NumPy copy of a CuPy/torch/NumPy array or a scalar."""
    if hasattr(a, "get"):
        return np.asarray(a.get())
    if hasattr(a, "detach"):
        return a.detach().cpu().numpy()
    return np.asarray(a)


_TYPESTR = {"fp64": "<f8", "fp32": "<f4"}


def _ptr(a, what, kind="field", count=None):
    """Device address of `a` after checking its element type and contiguity."""
    if a is None:
        return None
    try:
        ai = a.__cuda_array_interface__
    except AttributeError:
        raise SailfishError("%s: not a CUDA array (no __cuda_array_interface__)" % what)
    want = {"field": _TYPESTR[_prec], "acc": "<f8", "int": "<i4"}[kind]
    if ai["typestr"] != want:
        raise SailfishError("%s: element type %s, expected %s" % (what, ai["typestr"], want))
    shape = tuple(ai["shape"])
    st = ai.get("strides")
    if st is not None:
        esz = int(want[2])
        exp, acc = [], esz
        for s_ in reversed(shape):
            exp.append(acc)
            acc *= s_
        if tuple(reversed(exp)) != tuple(st) and int(np.prod(shape)) > 1:
            raise SailfishError("%s: not C-contiguous" % what)
    n = int(np.prod(shape)) if shape else 1
    if count is not None and n < count:
        raise SailfishError("%s: %d elements, at least %d needed" % (what, n, count))
    return ctypes.c_void_p(ai["data"][0])


def _need():
    if _ctx is None:
        raise SailfishError("initModule(GRID, BOUNDARY) has not been called")
    return _ctx


def initModule(GRID, BOUNDARY=None, precision="fp64"):
    """Grid metrics, S-coordinate tables and boundary programs into a device context on the
    current CUDA device (modules/mod_operators.py:31-45 with the index setup of
    modules/mod_boundary.py:237-297).  BOUNDARY may be the reference's Boundary or None (the
    reference's default lateral boundary conditions are then built here)."""
    global _ctx, _prec
    L, M, N = int(GRID.L), int(GRID.M), int(GRID.N)
    g = Grid(L, M, N, *(_host(getattr(GRID, k)) for k in
                        ("h", "pm", "pn", "on_u", "om_v", "fomn", "sc_r", "sc_w", "Cs_r", "Cs_w")),
             float(_host(GRID.hc)), int(_host(GRID.Vtransform)))
    B = BOUNDARY if BOUNDARY is not None else host.Boundary(L, M)
    _HostBoundary.check(B)
    if _ctx is not None:
        _ctx.close()
    _ctx = Context(g, _HostBoundary(B), precision)
    _prec = precision
    return _ctx


class _HostBoundary:
    """Boundary index arrays on the host, from the reference's Boundary (CuPy or NumPy)."""

    FIELDS = ("zetaClosedOrGradientBCIdx1", "zetaClosedOrGradientBCIdx2", "zetaClampedBCIdx1",
              "ubarClosedBCIdx1", "vbarClosedBCIdx1", "ubarClampedBCIdx1", "vbarClampedBCIdx1",
              "ubarGradientBCIdx1", "ubarGradientBCIdx2", "vbarGradientBCIdx1",
              "vbarGradientBCIdx2")

    class _BC:
        pass

    def __init__(self, B):
        for f in self.FIELDS:
            setattr(self, f, _host(getattr(B, f)))
        for name in ("zetaBC", "ubarBC", "vbarBC", "uvelBC", "vvelBC"):
            src, dst = getattr(B, name), self._BC()
            for f in ("bcIdxFieldIdx2", "bcIdxFieldType"):
                setattr(dst, f, _host(getattr(src, f)))
            setattr(self, name, dst)

    @classmethod
    def check(cls, B):
        missing = [f for f in cls.FIELDS if not hasattr(B, f)]
        if missing:
            raise SailfishError("BOUNDARY lacks %s" % ", ".join(missing))


def _state(OCEAN):
    s = State2D()
    for n in ("zeta", "ubar", "vbar", "rzeta", "rubar", "rvbar"):
        arr = getattr(s, n)
        for k in range(3):
            arr[k] = _ptr(getattr(OCEAN, "%s_t%d" % (n, k)), "%s_t%d" % (n, k)).value
    s.Zt_avg1 = _ptr(OCEAN.Zt_avg1, "Zt_avg1", "acc").value
    s.DU_avg1 = _ptr(OCEAN.DU_avg1, "DU_avg1", "acc").value
    s.DV_avg1 = _ptr(OCEAN.DV_avg1, "DV_avg1", "acc").value
    return s


# ---- step2d -------------------------------------------------------------------------------
def step2dPredictor(compTimes, GRID, OCEAN, BOUNDARY):
    c = _need()
    s = _state(OCEAN)
    check(lib.sf_step2d_predictor(c.ptr, ctypes.byref(s), float(compTimes.dtfast),
                                  float(compTimes.time2D), int(bool(compTimes.isFirst2DStep())),
                                  stream), "step2dPredictor")


def step2dCorrector(compTimes, GRID, OCEAN, BOUNDARY):
    c = _need()
    s = _state(OCEAN)
    cff1 = float(_host(compTimes.weight1)[compTimes.iif - 1])
    check(lib.sf_step2d_corrector(c.ptr, ctypes.byref(s), float(compTimes.dtfast),
                                  float(compTimes.time2D), cff1, stream), "step2dCorrector")


def zetabc(zeta, compTimes, BOUNDARY):
    check(lib.sf_zetabc(_need().ptr, _ptr(zeta, "zeta"), stream), "zetabc")


def barotropicVelocityBC(ubar, vbar, compTimes, BOUNDARY):
    check(lib.sf_barotropic_velocity_bc(_need().ptr, _ptr(ubar, "ubar"), _ptr(vbar, "vbar"),
                                        float(compTimes.time2D), stream), "barotropicVelocityBC")


# ---- rhs3d ---------------------------------------------------------------------------------
def rhs3d(GRID, OCEAN, BOUNDARY):
    c = _need()
    n3 = (c.grid.N + 1) * c.grid.s2
    check(lib.sf_rhs3d(c.ptr, _ptr(OCEAN.u_t2, "u_t2", count=n3), _ptr(OCEAN.v_t2, "v_t2", count=n3),
                       _ptr(OCEAN.Huon, "Huon", count=n3), _ptr(OCEAN.Hvom, "Hvom", count=n3),
                       _ptr(OCEAN.W, "W", count=n3), _ptr(GRID.Hz, "Hz"),
                       _ptr(OCEAN.ru_t2, "ru_t2", count=n3), _ptr(OCEAN.rv_t2, "rv_t2", count=n3),
                       stream), "rhs3d")


# ---- RawKernel-style callables ------------------------------------------------------------
class _Kernel:
    """A callable with the reference's RawKernel convention kernel(grid, block, args)."""

    def __init__(self, name, fn):
        self.name, self.fn = name, fn

    def __call__(self, grid=None, block=None, args=None):
        if args is None and isinstance(grid, tuple) and block is None:
            args = grid             # kernel(args) also accepted
        return self.fn(*args)


def _set_maxflux(u, v, Huon, Hvom, Hz):
    check(lib.sf_set_maxflux(_need().ptr, _ptr(u, "u"), _ptr(v, "v"), _ptr(Huon, "Huon"),
                             _ptr(Hvom, "Hvom"), _ptr(Hz, "Hz"), stream), "set_maxflux")


def _omega(W, u, v, Huon, Hvom, z_w, BC):
    check(lib.sf_omega(_need().ptr, _ptr(W, "W"), _ptr(Huon, "Huon"), _ptr(Hvom, "Hvom"),
                       _ptr(z_w, "z_w"), stream), "omega")


def _set_zeta(zeta_t1, zeta_t2, Zt_avg1):
    check(lib.sf_set_zeta(_need().ptr, _ptr(zeta_t1, "zeta_t1"), _ptr(zeta_t2, "zeta_t2"),
                          _ptr(Zt_avg1, "Zt_avg1", "acc"), stream), "set_zeta")


def _set_depth(Vtransform, Zt_avg1, z_w, z_r, h, hc, Hz, sc_r, sc_w, Cs_r, Cs_w):
    c = _need()
    if int(Vtransform) != c.grid.Vtransform:
        raise SailfishError("set_depth: Vtransform %d, the module was initialised with %d"
                            % (int(Vtransform), c.grid.Vtransform))
    check(lib.sf_set_depth(c.ptr, _ptr(Zt_avg1, "Zt_avg1", "acc"), _ptr(z_w, "z_w"),
                           _ptr(z_r, "z_r"), _ptr(Hz, "Hz"), stream), "set_depth")


def _step3d_UV(u, v, ru, rv, ubar_t1, vbar_t1, ubar_t2, vbar_t2, Hz, AKv, z_r, DU_avg1,
               DV_avg1, tmpU, tmpV, h, iic, ntfirst, lam, AK, dt):
    check(lib.sf_step3d_uv(_need().ptr, _ptr(u, "u"), _ptr(v, "v"), _ptr(ru, "ru"), _ptr(rv, "rv"),
                           _ptr(ubar_t1, "ubar_t1"), _ptr(vbar_t1, "vbar_t1"),
                           _ptr(ubar_t2, "ubar_t2"), _ptr(vbar_t2, "vbar_t2"), _ptr(Hz, "Hz"),
                           _ptr(AKv, "AKv"), _ptr(z_r, "z_r"), _ptr(DU_avg1, "DU_avg1", "acc"),
                           _ptr(DV_avg1, "DV_avg1", "acc"), _ptr(tmpU, "tmpU"),
                           _ptr(tmpV, "tmpV"), int(iic), int(ntfirst), float(lam), float(dt),
                           stream), "step3d_UV")


def _setLateralUVBCs(time, u, v, uIdx, vIdx, uType, vType):
    check(lib.sf_lateral_uv_bc(_need().ptr, float(time), _ptr(u, "u"), _ptr(v, "v"), stream),
          "setLateralUVBCs")


set_maxflux = _Kernel("set_maxflux", _set_maxflux)
omega = _Kernel("omega", _omega)
set_zeta = _Kernel("set_zeta", _set_zeta)
set_depth = _Kernel("set_depth", _set_depth)
step3d_UV = _Kernel("step3d_UV", _step3d_UV)
setLateralUVBCs = _Kernel("setLateralUVBCs", _setLateralUVBCs)


# ---- GLS ------------------------------------------------------------------------------------
GADV = 1.0 / 3.0   # third-order upstream-biased weight (gls_corrector_step.py:214-215, :236)


def gls_predictor_step(compTimes, GRID, OCEAN, MIXING):
    """GLS predictor (nonlinear/gls_predictor_step.py:18-216) on the reference's state objects.
    MIXING: tke, gls (time level nstp), optional tke_old/gls_old (level indx, the previous
    step's; the forward first step when absent or compTimes.iic == compTimes.ntfirst), and the
    caller's arrays tke_aux, gls_aux (time level 3), tke_nnew, gls_nnew and Hz_half, written
    here ((N+1) W levels each).  Huon, Hvom and W are OCEAN's, Hz is GRID's."""
    c = _need()
    old_t = getattr(MIXING, "tke_old", None)
    old_g = getattr(MIXING, "gls_old", None)
    first = (old_t is None or old_g is None or
             getattr(compTimes, "iic", 0) == getattr(compTimes, "ntfirst", 0))
    check(lib.sf_gls_predictor(
        c.ptr, float(compTimes.dt), int(first), _ptr(OCEAN.Huon, "Huon"),
        _ptr(OCEAN.Hvom, "Hvom"), _ptr(OCEAN.W, "W"), _ptr(GRID.Hz, "Hz"),
        _ptr(MIXING.tke, "tke"), _ptr(MIXING.tke if first else old_t, "tke_old"),
        _ptr(MIXING.tke_aux, "tke_aux"), _ptr(MIXING.tke_nnew, "tke_nnew"),
        _ptr(MIXING.gls, "gls"), _ptr(MIXING.gls if first else old_g, "gls_old"),
        _ptr(MIXING.gls_aux, "gls_aux"), _ptr(MIXING.gls_nnew, "gls_nnew"),
        _ptr(MIXING.Hz_half, "Hz_half"), stream), "gls_predictor_step")


def gls_corrector_step(compTimes, GRID, OCEAN, MIXING, FORCES):
    """GLS corrector on the reference's state objects.  MIXING: tke, gls, Akt, Akk, Akp,
    Lscale and bvf ((N+1) W levels each), optional `params` (a GlsParams, or the name of a
    model in closure.GLS_PRESETS: "k-epsilon" (the default), "k-omega", "gen"/"k-psi");
    Akv is OCEAN.AKv.  FORCES: sustr, svstr (kinematic surface stress at U/V points).  u, v
    are OCEAN.u_t2/v_t2; z_r and Hz come from GRID.  When MIXING holds tke_nnew (after
    gls_predictor_step), the new level is first advected (gls_corrector_step.py:172-388, with
    MIXING.gadv, default 1/3, and OCEAN's Huon, Hvom, W) and the corrector starts from it;
    otherwise it starts from Hz_w * tke (no advection)."""
    from .closure import GLS_PRESETS, gls_defaults, gls_preset
    c = _need()
    P = getattr(MIXING, "params", None) or gls_defaults()
    if isinstance(P, str):
        if P not in GLS_PRESETS:
            raise SailfishError("MIXING.params: GLS model must be one of %s" % sorted(GLS_PRESETS))
        P = gls_preset(P)
    if not isinstance(P, GlsParams):
        raise SailfishError("MIXING.params must be a GlsParams or a GLS model name")
    if getattr(MIXING, "tke_nnew", None) is not None:
        # after gls_predictor_step: advect the new level, then start the corrector from it
        check(lib.sf_gls_advect(
            c.ptr, ctypes.byref(P), float(compTimes.dt), float(getattr(MIXING, "gadv", GADV)),
            _ptr(OCEAN.Huon, "Huon"), _ptr(OCEAN.Hvom, "Hvom"), _ptr(OCEAN.W, "W"),
            _ptr(MIXING.tke_aux, "tke_aux"), _ptr(MIXING.gls_aux, "gls_aux"),
            _ptr(MIXING.tke_nnew, "tke_nnew"), _ptr(MIXING.gls_nnew, "gls_nnew"), stream),
            "gls_corrector_step")
        check(lib.sf_gls_corrector_nnew(
            c.ptr, ctypes.byref(P), float(compTimes.dt), _ptr(OCEAN.u_t2, "u_t2"),
            _ptr(OCEAN.v_t2, "v_t2"), _ptr(GRID.z_r, "z_r"), _ptr(GRID.Hz, "Hz"),
            _ptr(MIXING.bvf, "bvf"), _ptr(FORCES.sustr, "sustr"), _ptr(FORCES.svstr, "svstr"),
            _ptr(MIXING.tke_nnew, "tke_nnew"), _ptr(MIXING.gls_nnew, "gls_nnew"),
            _ptr(MIXING.tke, "tke"), _ptr(MIXING.gls, "gls"), _ptr(OCEAN.AKv, "AKv"),
            _ptr(MIXING.Akt, "Akt"), _ptr(MIXING.Akk, "Akk"), _ptr(MIXING.Akp, "Akp"),
            _ptr(MIXING.Lscale, "Lscale"), stream), "gls_corrector_step")
        return
    check(lib.sf_gls_corrector(
        c.ptr, ctypes.byref(P), float(compTimes.dt), _ptr(OCEAN.u_t2, "u_t2"),
        _ptr(OCEAN.v_t2, "v_t2"), _ptr(GRID.z_r, "z_r"), _ptr(GRID.Hz, "Hz"),
        _ptr(MIXING.bvf, "bvf"), _ptr(FORCES.sustr, "sustr"), _ptr(FORCES.svstr, "svstr"),
        _ptr(MIXING.tke, "tke"), _ptr(MIXING.gls, "gls"), _ptr(OCEAN.AKv, "AKv"),
        _ptr(MIXING.Akt, "Akt"), _ptr(MIXING.Akk, "Akk"), _ptr(MIXING.Akp, "Akp"),
        _ptr(MIXING.Lscale, "Lscale"), stream), "gls_corrector_step")
