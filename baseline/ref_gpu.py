"""The reference's own CUDA kernels on the GPU, launched in its main3d order: the plain FP64
GPU step that the FP32 form is compared with.

The reference compiles its kernel sources at import time with NVRTC (CuPy RawModule,
modules/mod_operators.py:125-185) with the options ('-default-device', '--restrict',
'--std=c++17') of utility/misc.py:9, after renaming its Greek identifiers
(mod_operators.py:132-136), and launches them from Python (nonlinear/main3d.py:118-324,
nonlinear/step2d.py:23-128, nonlinear/rhs.py:16-93, zetabc.py, barotropicVelocityBC.py).
This module does the same without CuPy:

* ``generate()`` (a build recipe, run where the reference checkout is) writes the renamed
  sources to baseline/_ref/src; the stencil header's reference data members, which the
  reference binds to by-value constructor parameters (modules/mod_cppkernels.h:352,360 and
  the like: dangling references that only happen to work when everything is inlined), are
  declared by value, the value each reference aliases when it is bound; no expression,
  operand or order of evaluation changes.
* ``cubins()`` compiles them with NVRTC for sm_100a with the reference's options (cached as
  baseline/_ref/*.cubin; ``fmad=False`` adds --fmad=false, the contraction-free build that
  reproduces the IEEE evaluation of every expression as written).
* ``RefGPU`` loads the modules through the CUDA driver API, sets the device globals with the
  reference's ``initialize`` kernels, and runs main3d with the reference's launch geometry
  (grsz = s2/512 + 1 blocks of 512; the "x GPUMUL" launches grsz*2 blocks of 256,
  mod_operators.py:40-41, utility/misc.py:10,17) on fields it allocates itself.  The
  reference's CuPy array operations (ru[:] = 0, the accumulator resets, vbar_t2[:] = 0, the
  tmpU/tmpV copies) are device memsets and copies.

Every field lives at offset G = s2 + 4 I + 1024 elements inside a zero-filled parent of
n + 2 G elements: the reference's stencils read before and after its arrays at the boundary
ring (rhs_kernels.cpp:86-91 has no guard at all), and with the host-compiled kernels and the
same launch geometry every access was found to stay within G of its array (page fences
around the guards, square, non-square and odd grids).  The 3D velocities and tendencies
keep the reference's three-slot parents (mod_ocean.py:65-71), of which slot 2 is used.
"""
import ctypes
import os
import re
import sys
import unicodedata

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
SRC = os.path.join(OUT, "src")
MODULES = {"2d": "modules/mod_cppkernels.cpp", "rhs": "nonlinear/rhs_kernels.cpp",
           "step3d": "nonlinear/step3D_uv.kernels.cpp", "bc": "modules/mod_BC.c"}
OPTIONS = ("-default-device", "--restrict", "--std=c++17")     # utility/misc.py:9
G_GRAV = 10.0                                                    # modules/mod_constants.py:26
BC_OMEGA = 0.0002                                                # barotropicVelocityBC.py:21-24


def reference_root():
    return os.environ.get("SAILFISH_REFERENCE",
                          os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))


def _rename(code):   # modules/mod_operators.py:132-136
    for a, b in (("η", "E"), ("ξ", "X"), ("Δ", "D"), ("σ", "sig")):
        code = code.replace(a, b)
    return unicodedata.normalize("NFKD", code).encode("ascii", "ignore").decode("ascii")


def generate(verbose=False):
    """Build recipe: the reference's kernel sources, renamed as its loader renames them, into
    baseline/_ref/src.  Returns False where the reference checkout is absent."""
    ref = reference_root()
    if not os.path.isdir(ref):
        return False
    os.makedirs(SRC, exist_ok=True)
    with open(os.path.join(ref, "modules", "mod_cppkernels.h"), encoding="utf-8-sig") as f:
        hdr = _rename(f.read())
    hdr = re.sub(r"^(\s*)(L|R|OType) &(\w+);", r"\1\2 \3;", hdr, flags=re.M)
    _write_if_changed(os.path.join(SRC, "mod_cppkernels.h"), hdr)
    for name, rel in MODULES.items():
        with open(os.path.join(ref, rel), encoding="utf-8-sig") as f:
            code = _rename(f.read())
        _write_if_changed(os.path.join(SRC, name + ".cu"), code)
        if verbose:
            print("baseline/_ref/src/%s.cu <- %s" % (name, rel))
    return True


def _write_if_changed(path, text):
    if os.path.exists(path):
        with open(path) as f:
            if f.read() == text:
                return
    with open(path, "w") as f:
        f.write(text)


def available():
    return all(os.path.exists(os.path.join(SRC, n + ".cu")) for n in MODULES)


def _nvrtc_check(res, prog=None):
    from cuda.bindings import nvrtc
    err = res[0]
    if err != nvrtc.nvrtcResult.NVRTC_SUCCESS:
        log = ""
        if prog is not None:
            _, n = nvrtc.nvrtcGetProgramLogSize(prog)
            buf = b" " * n
            nvrtc.nvrtcGetProgramLog(prog, buf)
            log = buf.decode(errors="replace")
        raise RuntimeError("NVRTC: %s\n%s" % (err, log))
    return res[1:] if len(res) > 2 else (res[1] if len(res) == 2 else None)


def cubins(fmad=True, verbose=False):
    """{module: cubin bytes} for sm_100a, compiled by NVRTC with the reference's options (and
    --fmad=false when fmad is False), cached in baseline/_ref."""
    from cuda.bindings import nvrtc
    if not available():
        raise RuntimeError("baseline/_ref/src is missing: run python baseline/ref_gpu.py where "
                           "the reference checkout is present")
    with open(os.path.join(SRC, "mod_cppkernels.h")) as f:
        hdr = f.read().encode()
    out = {}
    for name in MODULES:
        path = os.path.join(OUT, "ref_%s%s.cubin" % (name, "" if fmad else "_nofma"))
        src = os.path.join(SRC, name + ".cu")
        hsrc = os.path.join(SRC, "mod_cppkernels.h")
        if (os.path.exists(path) and os.path.getmtime(path) >= os.path.getmtime(src)
                and os.path.getmtime(path) >= os.path.getmtime(hsrc)):
            with open(path, "rb") as f:
                out[name] = f.read()
            continue
        with open(src) as f:
            code = f.read().encode()
        prog = _nvrtc_check(nvrtc.nvrtcCreateProgram(code, (name + ".cu").encode(), 2,
                                                     [hdr, hdr],
                                                     [b"mod_cppkernels.h", b"./mod_cppkernels.h"]))
        opts = [o.encode() for o in OPTIONS] + [b"-arch=sm_100a"] + ([] if fmad else [b"--fmad=false"])
        res = nvrtc.nvrtcCompileProgram(prog, len(opts), opts)
        _nvrtc_check((res[0], None), prog)
        size = _nvrtc_check(nvrtc.nvrtcGetCUBINSize(prog))
        buf = b" " * size
        _nvrtc_check((nvrtc.nvrtcGetCUBIN(prog, buf)[0], None))
        nvrtc.nvrtcDestroyProgram(prog)
        with open(path, "wb") as f:
            f.write(buf)
        if verbose:
            print("NVRTC %s -> %s (%d bytes)" % (name, path, size))
        out[name] = buf
    return out


# argument types of each kernel (in the reference's parameter order)
_P, _D, _I, _U, _B = "p", "d", "i", "u", "b"
SIGS = {
    "2d": {"initialize": [_U, _U, _U] + [_P] * 4,
           "computeMomentumRHSPred": [_P] * 5 + [_D, _D],
           "computeMomentumRHSCorr": [_P] * 6 + [_D],
           "computeZetaRHS": [_P] * 7 + [_B, _P, _P, _I, _P],
           "computeZetaPred": [_D] + [_P] * 4,
           "computeMomentumPred": [_D] + [_P] * 9,
           "AdamsMoultonCorr3rd": [_D] + [_P] * 4},
    "rhs": {"initialize": [_U, _U, _U] + [_P] * 4,
            "addCoriolis": [_P] * 6, "horizontalAdvection": [_P] * 7,
            "verticalAdvection": [_P] * 6},
    "step3d": {"initialize": [_U, _U, _U] + [_P] * 4, "setVerticalVelEq": [_P] * 3,
               "omega": [_P] * 7, "set_depth": [_I] + [_P] * 4 + [_D] + [_P] * 5,
               "set_zeta": [_P] * 3, "setLateralUVBCs": [_D] + [_P] * 6,
               "set_maxflux": [_P] * 5, "step3d_UV": [_P] * 16 + [_I, _I, _D, _D, _D]},
    "bc": {"setBC": [_P, _P, _U, _D], "copyBC": [_P, _P, _P, _U]},
}
_CT = {_P: ctypes.c_void_p, _D: ctypes.c_double, _I: ctypes.c_int, _U: ctypes.c_uint,
       _B: ctypes.c_bool}


class RefGPU:
    """The reference's time step on the current CUDA device (torch's current stream)."""

    def __init__(self, b, nfast, weight1, weight2, fmad=True, init=None):
        """b: a basin dict (L, M, N, h, pm, pn, on_u, om_v, fomn, sc_r, sc_w, Cs_r, Cs_w, hc,
        Vtransform, dt, ndtfast, lists) as the oracle's set-up builds it; init: optional
        {name: host array} of initial fields (u, v, ru, rv as (N+1, M+1, L+1) slot-2 values)."""
        import numpy as np
        import torch
        from cuda.bindings import driver as drv
        self.np, self.torch, self.drv = np, torch, drv
        self.dev = torch.device("cuda", torch.cuda.current_device())
        # the driver-API module loads need the device's primary context current on this thread
        torch.zeros(1, device=self.dev)
        torch.cuda.synchronize()
        self.funcs = {}
        self.mods = []
        for name, cubin in cubins(fmad).items():
            err, mod = drv.cuModuleLoadData(cubin)
            if err != drv.CUresult.CUDA_SUCCESS:
                raise RuntimeError("cuModuleLoadData(%s): %s" % (name, err))
            self.mods.append(mod)
            for fn in SIGS[name]:
                err, f = drv.cuModuleGetFunction(mod, fn.encode())
                if err != drv.CUresult.CUDA_SUCCESS:
                    raise RuntimeError("cuModuleGetFunction(%s): %s" % (fn, err))
                self.funcs[(name, fn)] = f
        L, M, N = b["L"], b["M"], b["N"]
        I, J = L + 1, M + 1
        self.L, self.M, self.N, self.I, self.J, self.s2 = L, M, N, I, J, I * J
        self.G = self.s2 + 4 * I + 1024
        self.keep = []
        f64 = torch.float64
        g = lambda a: self._put(np.asarray(a, np.float64).ravel(), f64)
        self.h, self.pm, self.pn, self.on_u, self.om_v, self.fomn = (
            g(b[k]) for k in ("h", "pm", "pn", "on_u", "om_v", "fomn"))
        self.sc_r, self.sc_w, self.Cs_r, self.Cs_w = (g(b[k]) for k in ("sc_r", "sc_w", "Cs_r", "Cs_w"))
        self.hc, self.Vtransform = float(b["hc"]), int(b["Vtransform"])
        s2, n3 = self.s2, (N + 1) * self.s2
        z = lambda n: self._zeros(n, f64)
        for k in ("zeta", "ubar", "vbar", "rzeta", "rubar", "rvbar"):
            setattr(self, k, z(3 * s2))
        self.slots = {k: [0, 1, 2] for k in ("zeta", "ubar", "vbar", "rzeta", "rubar", "rvbar")}
        for k in ("u", "v", "ru", "rv"):        # (3, N+1, J, I) parents, slot 2 used
            setattr(self, k, z(3 * n3))
        for k in ("W", "Huon", "Hvom", "AKv", "z_w", "eqSD", "eqD", "eqRHS", "tmpU", "tmpV"):
            setattr(self, k, z(n3))
        for k in ("z_r", "Hz"):
            setattr(self, k, z(N * s2))
        for k in ("Zt_avg1", "DU_avg1", "DV_avg1"):
            setattr(self, k, z(s2))
        self.AKv.fill_(0.001)                   # modules/mod_ocean.py:91
        self.w1 = self._put(np.asarray(weight1, np.float64), f64)
        self.w2 = self._put(np.asarray(weight2, np.float64), f64)
        lists = b["lists"]
        self.B = {k: self._put(np.asarray(v, np.int32).ravel(), torch.int32) for k, v in lists.items()}
        self.nB = {k: int(np.asarray(v).size) for k, v in lists.items()}
        self.dt, self.ndtfast = float(b["dt"]), int(b["ndtfast"])
        self.dtfast = self.dt / self.ndtfast
        self.nfast = int(nfast)
        self.iic, self.iif, self.ntfirst = 0, 0, 0
        self.time, self.time2D = 0.0, 0.0
        if init:
            for k, a in init.items():
                a = np.asarray(a, np.float64)
                if k in ("u", "v", "ru", "rv"):
                    self.t3(k).copy_(torch.from_numpy(a.ravel()))
                elif k in self.slots:
                    getattr(self, k).copy_(torch.from_numpy(a.ravel()))
                else:
                    getattr(self, k).copy_(torch.from_numpy(a.ravel()))
        self.nt = (s2 // 512 + 1) * 512          # grsz*bksz = grsz*GPUMUL*(bksz/GPUMUL)
        self.grsz = s2 // 512 + 1
        for mod in ("2d", "rhs", "step3d"):
            self.launch(mod, "initialize", 1, 1, N, J, I, self.on_u, self.om_v, self.pn, self.pm)
        self.launch("step3d", "setVerticalVelEq", 1, 1, self.eqSD, self.eqD, self.eqRHS)
        self.started = False

    # -- memory ---------------------------------------------------------------------------
    def _zeros(self, n, dtype):
        t = self.torch.zeros(n + 2 * self.G, dtype=dtype, device=self.dev)
        self.keep.append(t)
        return t[self.G:self.G + n]

    def _put(self, a, dtype):
        t = self._zeros(a.size, dtype)
        t.copy_(self.torch.from_numpy(a))
        return t

    def t(self, name, k):         # 2D slot k (t0, t1, t2) of a three-level field
        return getattr(self, name)[self.slots[name][k] * self.s2:(self.slots[name][k] + 1) * self.s2]

    def t3(self, name):           # slot 2 of a 3D parent
        n3 = (self.N + 1) * self.s2
        return getattr(self, name)[2 * n3:3 * n3]

    def cycle2d(self):            # T_OCEAN.cycleTimes2D (mod_ocean.py:120-154)
        for k, s in self.slots.items():
            self.slots[k] = [s[1], s[2], s[0]]

    # -- launches -------------------------------------------------------------------------
    def launch(self, mod, fn, grid, block, *args):
        types = SIGS[mod][fn]
        objs = []
        for t, a in zip(types, args):
            if t == _P:
                objs.append(ctypes.c_void_p(a.data_ptr() if hasattr(a, "data_ptr") else int(a)))
            else:
                objs.append(_CT[t](a))
        arr = (ctypes.c_void_p * len(objs))(*[ctypes.addressof(o) for o in objs])
        stream = self.torch.cuda.current_stream().cuda_stream
        err, = self.drv.cuLaunchKernel(self.funcs[(mod, fn)], grid, 1, 1, block, 1, 1, 0, stream,
                                       ctypes.addressof(arr), 0)
        if err != self.drv.CUresult.CUDA_SUCCESS:
            raise RuntimeError("cuLaunchKernel(%s): %s" % (fn, err))

    def k(self, mod, fn, *args):              # grsz x bksz
        self.launch(mod, fn, self.grsz, 512, *args)

    def k2(self, mod, fn, *args):             # (grsz*GPUMUL,) x (bksz//GPUMUL,)
        self.launch(mod, fn, self.grsz * 2, 256, *args)

    def _set_bc(self, var, key, val):          # setBC (mod_BC.c:6)
        n = self.nB[key]
        if n:
            self.launch("bc", "setBC", n // 512 + 1, 512, var, self.B[key], n, val)

    def _copy_bc(self, var, k1, k2, n):        # copyBC (mod_BC.c:16)
        if n:
            self.launch("bc", "copyBC", n // 512 + 1, 512, var, self.B[k1], self.B[k2], n)

    def zetabc(self, z):                       # nonlinear/zetabc.py:5-12
        self._copy_bc(z, "zetaClosedOrGradientBCIdx1", "zetaClosedOrGradientBCIdx2",
                      self.nB["zetaClosedOrGradientBCIdx1"])

    def velbc(self, ub, vb):                   # nonlinear/barotropicVelocityBC.py:7-31
        import math
        self._set_bc(ub, "ubarClosedBCIdx1", 0.0)
        self._set_bc(vb, "vbarClosedBCIdx1", 0.0)
        self._set_bc(ub, "ubarClampedBCIdx1", .05 * math.sin(self.time2D * BC_OMEGA))
        self._copy_bc(ub, "ubarGradientBCIdx1", "ubarGradientBCIdx2", self.nB["ubarGradientBCIdx1"])
        self._copy_bc(vb, "vbarGradientBCIdx1", "ubarGradientBCIdx2", self.nB["vbarGradientBCIdx1"])

    # -- the step -------------------------------------------------------------------------
    def set_depth(self):                       # main3d.py:62,290
        self.k("step3d", "set_depth", self.Vtransform, self.Zt_avg1, self.z_w, self.z_r, self.h,
               self.hc, self.Hz, self.sc_r, self.sc_w, self.Cs_r, self.Cs_w)

    def predictor(self):                       # nonlinear/step2d.py:23-81 (leapfrog branch)
        t = self.t
        self.k2("2d", "computeZetaRHS", t("zeta", 1), self.h, t("ubar", 1), t("vbar", 1),
                self.DU_avg1, self.DV_avg1, self.Zt_avg1, True, self.w1, self.w2, self.iif,
                t("rzeta", 1))
        self.k("2d", "computeZetaPred", self.dtfast, t("zeta", 0), t("zeta", 1), t("zeta", 2),
               t("rzeta", 1))
        self.zetabc(t("zeta", 2))
        self.k("2d", "computeMomentumRHSPred", self.h, t("rubar", 1), t("rvbar", 1), t("zeta", 0),
               t("zeta", 2), G_GRAV, 2.0 / 5.0)
        self.k("2d", "computeMomentumPred", self.dtfast, t("ubar", 1), t("ubar", 2), t("vbar", 1),
               t("vbar", 2), t("rubar", 1), t("rvbar", 1), self.h, t("zeta", 1), t("zeta", 2))
        self.velbc(t("ubar", 2), t("vbar", 2))

    def corrector(self):                       # nonlinear/step2d.py:84-128
        t = self.t
        self.k2("2d", "computeZetaRHS", t("zeta", 2), self.h, t("ubar", 2), t("vbar", 2),
                self.DU_avg1, self.DV_avg1, self.Zt_avg1, False, self.w1, self.w2, self.iif,
                t("rzeta", 1))
        self.k("2d", "AdamsMoultonCorr3rd", self.dtfast, t("zeta", 2), t("rzeta", 0),
               t("rzeta", 1), t("rzeta", 2))
        self.zetabc(t("zeta", 2))
        self.k("2d", "computeMomentumRHSCorr", self.h, t("rubar", 2), t("rvbar", 2), t("zeta", 0),
               t("zeta", 1), t("zeta", 2), G_GRAV)
        # AdamsMoultonCorr3rd2 is bound to AdamsMoultonCorr3rd (mod_operators.py:146): the
        # 5-argument kernel reads the first five of the 12 arguments step2d.py:120 passes
        self.k("2d", "AdamsMoultonCorr3rd", self.dtfast, t("ubar", 1), t("vbar", 1),
               t("rubar", 0), t("rubar", 1))
        self.velbc(t("ubar", 2), t("vbar", 2))

    def step(self, nsteps=1, lam=1.0, AK=1e-5, mixing=None):
        """main3d.py:118-324 for nsteps baroclinic steps; mixing(self), if given, runs after
        setLateralUVBCs (the reference's step has none)."""
        BC = self.B["zetaBC_bcIdxFieldIdx2"]
        if not self.started:
            self.set_depth()
            self.started = True
        for _ in range(nsteps):
            u, v, ru, rv = self.t3("u"), self.t3("v"), self.t3("ru"), self.t3("rv")
            self.k("step3d", "set_maxflux", u, v, self.Huon, self.Hvom, self.Hz)
            self.k("step3d", "omega", self.W, u, v, self.Huon, self.Hvom, self.z_w, BC)
            self.k("step3d", "set_zeta", self.t("zeta", 1), self.t("zeta", 2), self.Zt_avg1)
            ru.zero_()                                           # rhs.py:38-40
            rv.zero_()
            self.k("rhs", "addCoriolis", self.fomn, u, v, ru, rv, self.Hz)
            self.k2("rhs", "horizontalAdvection", u, v, self.Huon, self.Hvom, ru, rv, BC)
            self.k2("rhs", "verticalAdvection", u, v, self.W, ru, rv, BC)
            self.iif = 0
            for _ in range(self.nfast + 1):                      # main3d.py:166-189
                if self.iif == 0:
                    self.Zt_avg1.zero_()
                    self.DU_avg1.zero_()
                    self.DV_avg1.zero_()
                self.iif += 1                                    # next2DTimeStep
                self.time2D += self.dtfast
                self.cycle2d()
                self.predictor()
                self.corrector()
                self.t("vbar", 2).zero_()
            self.set_depth()
            self.tmpU.copy_(u)
            self.tmpV.copy_(v)
            self.k2("step3d", "step3d_UV", u, v, ru, rv, self.t("ubar", 1), self.t("vbar", 1),
                    self.t("ubar", 2), self.t("vbar", 2), self.Hz, self.AKv, self.z_r,
                    self.DU_avg1, self.DV_avg1, self.tmpU, self.tmpV, self.h, self.iic,
                    self.ntfirst, lam, AK, self.dt)
            self.k("step3d", "setLateralUVBCs", self.time, u, v, self.B["uvelBC_bcIdxFieldIdx2"],
                   self.B["vvelBC_bcIdxFieldIdx2"], self.B["uvelBC_bcIdxFieldType"],
                   self.B["vvelBC_bcIdxFieldType"])
            if mixing is not None:
                mixing(self)
            self.k("step3d", "omega", self.W, u, v, self.Huon, self.Hvom, self.z_w, BC)
            self.iic += 1                                        # nextTimeStep
            self.time += self.dt
            self.time2D = self.time

    def launches_per_step(self):
        """Kernel launches of one step (initialisation excluded), as the reference issues
        them: 3 + 3 (rhs3d) + per substep 5 + 5 (predictor, corrector) + the boundary
        scatters with entries, + set_depth, step3d_UV, setLateralUVBCs, omega."""
        bc_pred = 1 + sum(1 for k in ("ubarClosedBCIdx1", "vbarClosedBCIdx1", "ubarClampedBCIdx1",
                                      "ubarGradientBCIdx1", "vbarGradientBCIdx1") if self.nB[k])
        per_half = 4 + (1 if self.nB["zetaClosedOrGradientBCIdx1"] else 0) + bc_pred - 1
        return 3 + 3 + (self.nfast + 1) * 2 * per_half + 4


if __name__ == "__main__":
    ok = generate(verbose=True)
    if ok:
        for fm in (True, False):
            cubins(fm, verbose=True)
    sys.exit(0)
