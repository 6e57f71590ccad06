"""Device model: grid context, ocean state in HBM and the baroclinic step driver.

``Model.step()`` runs one step of the reference's 3D driver (nonlinear/main3d.py:118-324):

    set_maxflux + omega + set_zeta      sf_maxflux_omega        (main3d.py:118-151)
    rhs3d                               sf_rhs3d                (main3d.py:159, rhs.py:16-93)
    barotropic loop, nfast+1 substeps   sf_barotropic_loop      (main3d.py:166-189)
    set_depth                           sf_set_depth            (main3d.py:290)
    step3d_UV + setLateralUVBCs         sf_step3d_uv_bc         (main3d.py:304-311)
    vertical mixing (optional)          Model.mixing            (GLS or the learned closure)
    omega                               sf_omega                (main3d.py:321)

Layout in HBM: the reference's flat C-order fields.  The three barotropic time slots of each
2D field live in one (3, M+1, L+1) buffer and rotate by pointer (cycleTimes2D); the 3D
fields u, v, ru, rv keep only the slot the reference uses (its cycleTimes3D is never called,
so its other two slots are never read or written).
"""
import ctypes

import numpy as np
import torch

from . import host
from ._lib import lib, check, GridDesc, State2D, SF_FP64, SF_FP32

DTYPES = {"fp64": (SF_FP64, torch.float64, np.float64), "fp32": (SF_FP32, torch.float32, np.float32)}


def _i32(a):
    return np.ascontiguousarray(np.asarray(a).ravel(), dtype=np.int32)


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())


class Grid:
    """Horizontal grid, metrics and vertical coordinate (host FP64 arrays)."""

    def __init__(self, L, M, N, h, pm, pn, on_u, om_v, fomn, sc_r, sc_w, Cs_r, Cs_w, hc,
                 Vtransform):
        self.L, self.M, self.N = int(L), int(M), int(N)
        self.I, self.J = self.L + 1, self.M + 1
        self.s2 = self.I * self.J
        shp = (self.J, self.I)
        self.h, self.pm, self.pn, self.on_u, self.om_v, self.fomn = (
            np.asarray(a, np.float64).reshape(shp) for a in (h, pm, pn, on_u, om_v, fomn))
        self.sc_r, self.sc_w, self.Cs_r, self.Cs_w = (_f64(a) for a in (sc_r, sc_w, Cs_r, Cs_w))
        self.hc = float(hc)
        self.Vtransform = int(Vtransform)

    @classmethod
    def analytic(cls, Lm, Mm, N, h, dx, dy, f, Vtransform=2, Vstretching=4, theta_s=5.0,
                 theta_b=0.4, tcline=100.0):
        """Grid from rho-point depth h and Coriolis f ((Mm+2) x (Lm+2) arrays or scalars) on
        uniform spacing dx, dy, with the reference's metric and S-coordinate routines."""
        L, M = Lm + 1, Mm + 1
        shp = (M + 1, L + 1)
        h = np.broadcast_to(np.asarray(h, np.float64), shp).copy()
        f = np.broadcast_to(np.asarray(f, np.float64), shp).copy()
        pm = np.full(shp, 1.0 / dx)
        pn = np.full(shp, 1.0 / dy)
        m = host.update_metrics(pm, pn, f)
        sc_r, sc_w, Cs_r, Cs_w = host.set_coords(N, Vstretching, theta_s, theta_b)
        hc = min(h.min(), tcline) if Vtransform == 1 else tcline   # set_coords.py:355-359
        g = cls(L, M, N, h, pm, pn, m["on_u"], m["om_v"], m["fomn"], sc_r, sc_w, Cs_r, Cs_w, hc,
                Vtransform)
        g.f = f
        return g


def grid_desc(grid, boundary, precision, keep):
    """An sf_grid_desc for `grid` and `boundary`; the host arrays it points to are kept alive
    in the dict `keep`."""
    B = boundary

    def dp(name, a):
        keep[name] = _f64(a)
        return keep[name].ctypes.data_as(ctypes.POINTER(ctypes.c_double))

    def ip(name, a):
        keep[name] = _i32(a)
        return keep[name].ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), int(keep[name].size)

    d = GridDesc()
    d.L, d.M, d.N, d.precision = grid.L, grid.M, grid.N, DTYPES[precision][0]
    for k in ("h", "pm", "pn", "on_u", "om_v", "fomn", "sc_r", "sc_w", "Cs_r", "Cs_w"):
        setattr(d, k, dp(k, getattr(grid, k)))
    d.hc, d.Vtransform = grid.hc, grid.Vtransform
    d.zeta_field_idx2 = ip("zf", B.zetaBC.bcIdxFieldIdx2)[0]
    d.uvel_field_type = ip("ut", B.uvelBC.bcIdxFieldType)[0]
    d.vvel_field_type = ip("vt", B.vvelBC.bcIdxFieldType)[0]
    d.zeta_copy_idx1, d.n_zeta_copy = ip("z1", B.zetaClosedOrGradientBCIdx1)
    d.zeta_copy_idx2 = ip("z2", B.zetaClosedOrGradientBCIdx2)[0]
    d.ubar_closed_idx, d.n_ubar_closed = ip("uc", B.ubarClosedBCIdx1)
    d.vbar_closed_idx, d.n_vbar_closed = ip("vc", B.vbarClosedBCIdx1)
    d.ubar_clamped_idx, d.n_ubar_clamped = ip("ucl", B.ubarClampedBCIdx1)
    d.ubar_grad_idx1, d.n_ubar_grad = ip("ug1", B.ubarGradientBCIdx1)
    d.ubar_grad_idx2 = ip("ug2", B.ubarGradientBCIdx2)[0]
    d.vbar_grad_idx1, d.n_vbar_grad = ip("vg1", B.vbarGradientBCIdx1)
    return d


class Context:
    """An sf_ctx: the grid snapshot and boundary programs on the current CUDA device."""

    def __init__(self, grid, boundary, precision="fp64"):
        if precision not in DTYPES:
            raise ValueError("precision must be 'fp64' or 'fp32'")
        self.precision = precision
        self.grid = grid
        keep = {}
        d = grid_desc(grid, boundary, precision, keep)
        ptr = ctypes.c_void_p()
        check(lib.sf_ctx_create(ctypes.byref(d), ctypes.byref(ptr)), "sf_ctx_create")
        self.ptr = ptr

    def close(self):
        if getattr(self, "ptr", None):
            lib.sf_ctx_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def stream_handle():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class Model:
    """Ocean state in HBM and the reference's baroclinic step, run by libsailfish_b200."""

    NAMES2 = ("zeta", "ubar", "vbar", "rzeta", "rubar", "rvbar")
    NAMES3 = ("u", "v", "ru", "rv", "W", "Huon", "Hvom", "AKv")

    def __init__(self, grid, boundary, dt, ndtfast, precision="fp64", lam=1.0, device="cuda",
                 semantics="reference"):
        """semantics: "reference" (the reference's own step, bit-identical in FP64) or "roms"
        (the ROMS-form barotropic step with wind stress, quadratic bottom drag and Coriolis,
        surface stress on the 3D momentum and closed walls; set_forcing gives its stresses)."""
        if semantics not in ("reference", "roms"):
            raise ValueError("semantics must be 'reference' or 'roms'")
        self.semantics = semantics
        self.grid = grid
        self.ctx = Context(grid, boundary, precision)
        self.precision = precision
        self.tdtype = DTYPES[precision][1]
        self.dt, self.ndtfast = float(dt), int(ndtfast)
        self.dtfast = self.dt / self.ndtfast
        self.nfast, self.weight1, self.weight2 = host.set_weights(self.ndtfast)
        self._w1 = np.ascontiguousarray(self.weight1)
        self.lam = float(lam)
        self.iic, self.ntfirst = 0, 0
        self.time, self.time2D = 0.0, 0.0
        J, I, N = grid.J, grid.I, grid.N
        z = lambda *s, dt=None: torch.zeros(*s, dtype=dt or self.tdtype, device=device)
        for n in self.NAMES2:
            setattr(self, n, z(3, J, I))
        for n in self.NAMES3:
            setattr(self, n, z(N + 1, J, I))
        self.AKv.fill_(0.001)                     # modules/mod_ocean.py:91
        for n in ("Zt_avg1", "DU_avg1", "DV_avg1"):
            setattr(self, n, z(J * I, dt=torch.float64))
        self.z_w = z(N + 1, J, I)
        self.z_r = z(N, J, I)
        self.Hz = z(N, J, I)
        self.slots = [0, 1, 2]                    # (t0, t1, t2) rows of the 2D buffers
        self._started = False
        # vertical mixing per step (closure.Closure), after step3d_UV; None keeps AKv as it is,
        # as the reference's step does (modules/mod_ocean.py:91)
        self.mixing = None
        if semantics == "roms":
            # ROMS-indexed averaging weights, the second fast-time averages, the stresses
            self.W1, self.W2 = host.roms_weights(self.nfast, self.weight1)
            self.DU_avg2 = z(J * I, dt=torch.float64)
            self.DV_avg2 = z(J * I, dt=torch.float64)
            self.sustr = z(J * I)
            self.svstr = z(J * I)
            self.rdrag2 = 0.0
            # the 3D right-hand sides of steps n, n-1, n-2 (Adams-Bashforth), newest first;
            # self.ru / self.rv are the newest
            self._ru3 = [self.ru, z(N + 1, J, I), z(N + 1, J, I)]
            self._rv3 = [self.rv, z(N + 1, J, I), z(N + 1, J, I)]
        # blow-up check (sf_check_state) after every check_every-th step (0: never); a failed
        # check raises SailfishError with status SF_ENONFINITE
        self.check_every = 0
        self.surface_bound, self.velocity_bound = 100.0, 50.0

    # -- state I/O ------------------------------------------------------------------------
    def load(self, state):
        """Copy host arrays in the reference's shapes into the device state.  3D fields may be
        given as (3, N+1, M+1, L+1) parents, in which case their slot 2 is used."""
        for n, a in state.items():
            a = np.asarray(a)
            t = getattr(self, n)
            if n in ("u", "v", "ru", "rv") and a.ndim == 4:
                a = a[2]
            t.copy_(torch.from_numpy(np.ascontiguousarray(a).reshape(t.shape)).to(t.dtype))

    def state(self):
        out = {}
        for n in self.NAMES2 + self.NAMES3 + ("Zt_avg1", "DU_avg1", "DV_avg1", "z_w", "z_r", "Hz"):
            out[n] = getattr(self, n).double().cpu().numpy()
        out["slots"] = list(self.slots)
        return out

    # -- pointers ---------------------------------------------------------------------------
    def _p(self, t):
        return ctypes.c_void_p(t.data_ptr())

    def _slot(self, name, k):
        return getattr(self, name)[self.slots[k]]

    def state2d(self):
        s = State2D()
        for n in self.NAMES2:
            arr = getattr(s, n)
            for k in range(3):
                arr[k] = self._slot(n, k).data_ptr()
        s.Zt_avg1, s.DU_avg1, s.DV_avg1 = (self.Zt_avg1.data_ptr(), self.DU_avg1.data_ptr(),
                                           self.DV_avg1.data_ptr())
        return s

    def _sync_slots(self, s):
        base = {n: getattr(self, n).data_ptr() for n in self.NAMES2}
        row = self.grid.s2 * self.zeta.element_size()
        new = [(s.zeta[k] - base["zeta"]) // row for k in range(3)]
        for n in self.NAMES2[1:]:
            assert [(getattr(s, n)[k] - base[n]) // row for k in range(3)] == new
        self.slots = new

    # -- ROMS-form forcing -------------------------------------------------------------------
    def set_forcing(self, sustr=None, svstr=None, rdrag2=None):
        """Kinematic surface stress (m2/s2, (M+1)(L+1) arrays at U and V faces) and the
        quadratic bottom-drag coefficient of the ROMS-form step."""
        if self.semantics != "roms":
            raise ValueError("forcing applies to the ROMS-form step (semantics='roms')")
        for name, a in (("sustr", sustr), ("svstr", svstr)):
            if a is not None:
                getattr(self, name).copy_(torch.from_numpy(np.ascontiguousarray(a, np.float64).ravel()))
        if rdrag2 is not None:
            self.rdrag2 = float(rdrag2)

    def _roms_loop(self, s, stream):
        W1 = self.W1.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        W2 = self.W2.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        check(lib.sf_roms_barotropic_loop(
            self.ctx.ptr, ctypes.byref(s), self._p(self.DU_avg2), self._p(self.DV_avg2),
            self._p(self.sustr), self._p(self.svstr), self.rdrag2, self.nfast, W1, W2,
            self.dtfast, stream), "sf_roms_barotropic_loop")

    def step2d(self, nsteps=1, first=None):
        """2D-only steps of the ROMS-form scheme (predictor + corrector, no averages), the
        counterpart of the reference's main2d; the run's first step is forward/backward Euler."""
        if self.semantics != "roms":
            raise ValueError("step2d is the ROMS-form 2D driver (semantics='roms')")
        st = stream_handle()
        for _ in range(nsteps):
            f = (not getattr(self, "_started2d", False)) if first is None else first
            s = self.state2d()
            check(lib.sf_roms_step2d(self.ctx.ptr, ctypes.byref(s), self._p(self.sustr),
                                     self._p(self.svstr), self.rdrag2, self.dtfast, int(f), st),
                  "sf_roms_step2d")
            self._sync_slots(s)
            self._started2d = True
            self.time2D += self.dtfast

    # -- steps -------------------------------------------------------------------------------
    def check_state(self, stream=None):
        """Scans zeta/ubar/vbar (newest slot) and u, v for NaN, infinities and magnitudes above
        surface_bound / velocity_bound; raises SailfishError (SF_ENONFINITE) naming the first
        bad value.  Synchronises the stream."""
        st = stream or stream_handle()
        p = self._p
        check(lib.sf_check_state(self.ctx.ptr, p(self._slot("zeta", 2)), p(self._slot("ubar", 2)),
                                 p(self._slot("vbar", 2)), p(self.u), p(self.v),
                                 self.surface_bound, self.velocity_bound, st),
              "sf_check_state (step %d)" % self.iic)

    def set_depth(self, stream=None):
        st = stream or stream_handle()
        check(lib.sf_set_depth(self.ctx.ptr, self._p(self.Zt_avg1), self._p(self.z_w),
                               self._p(self.z_r), self._p(self.Hz), st), "sf_set_depth")

    def start(self):
        """main3d.py:62: depths from the initial Zt_avg1."""
        self.set_depth()
        self._started = True

    def _streams(self):
        """(loop, side, mix): a high-priority stream for the barotropic loop and two
        low-priority ones for rhs3d and the mixing, created once per model."""
        if getattr(self, "_strm", None) is None:
            lo, hi = torch.cuda.Stream.priority_range()
            dev = self.u.device
            self._strm = (torch.cuda.Stream(dev, priority=hi), torch.cuda.Stream(dev, priority=lo),
                          torch.cuda.Stream(dev, priority=lo))
        return self._strm

    def step(self, nsteps=1, final_omega=True, timer=None):
        """`nsteps` baroclinic steps (main3d.py:118-324).  The end-of-step omega
        (main3d.py:321) is recomputed at the start of every following step, so only the last
        one is evaluated unless `final_omega` is False (then none).  `timer(name)`, if given,
        returns a pair of CUDA events recorded around each phase (on the phase's stream).

        With `overlap` (off by default) the phases that share no field run concurrently: rhs3d
        (u, v, the fluxes, Hz -> ru, rv) beside the barotropic loop (2D state only), on their
        own streams (the loop's at high priority), both after set_maxflux/omega/set_zeta; and a
        mixing hook that declares `overlappable` (the package's closure: reads u, v, z_r, Hz,
        its own fields; writes AKv and its own fields) beside the next step's first phases,
        with set_depth (which rewrites z_r, Hz) and step3d (which reads AKv) waiting for it.
        Results are identical either way; the call returns with all its work queued on the
        current stream's order.  Measured on one B200 it does not pay: basin4 with the learned
        closure 11.85 ms per step sequential, 11.95 with the mixing overlapped, 13.04 with
        rhs3d beside the loop too (the closure's network holds a whole SM's shared memory and
        rhs3d its issue slots; the loop's short kernels lose more than is hidden); `overlap_rhs3d`
        = False keeps rhs3d in line."""
        if not self._started:
            self.start()
        c, p = self.ctx.ptr, self._p
        cs = torch.cuda.current_stream()
        st = ctypes.c_void_p(cs.cuda_stream)
        ovl = getattr(self, "overlap", False)
        ovl_rhs = ovl and getattr(self, "overlap_rhs3d", True)
        if ovl:
            s_loop, s_side, s_mix = self._streams()
        h = lambda strm: ctypes.c_void_p(strm.cuda_stream)
        mix_ovl = ovl and self.mixing is not None and getattr(self.mixing, "overlappable", False)
        ev_mix = None

        def phase(name, fn, strm=cs):
            if timer is None:
                return fn()
            a, b = timer(name)
            a.record(strm)
            r = fn()
            b.record(strm)
            return r

        def after(strm, *events):
            for e in events:
                if e is not None:
                    strm.wait_event(e)

        def mark(strm):
            e = torch.cuda.Event()
            e.record(strm)
            return e

        for k in range(nsteps):
            z1, z2 = self._slot("zeta", 1), self._slot("zeta", 2)
            phase("k_maxflux_omega", lambda: check(lib.sf_maxflux_omega(
                c, p(self.u), p(self.v), p(self.Huon), p(self.Hvom), p(self.Hz), p(self.W),
                p(self.z_w), p(z1), p(z2), p(self.Zt_avg1), st), "sf_maxflux_omega"))
            s = self.state2d()
            t2 = ctypes.c_double(self.time2D)
            rhs = lambda sh: check(lib.sf_rhs3d(
                c, p(self.u), p(self.v), p(self.Huon), p(self.Hvom), p(self.W), p(self.Hz),
                p(self.ru), p(self.rv), sh), "sf_rhs3d")
            loop = lambda sh: check(lib.sf_barotropic_loop(
                c, ctypes.byref(s), self.nfast + 1,
                self._w1.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), self.dtfast,
                ctypes.byref(t2), sh), "sf_barotropic_loop")
            if self.semantics == "roms":
                for r3 in (self._ru3, self._rv3):   # the oldest slot takes step n's
                    r3.insert(0, r3.pop())
                self.ru, self.rv = self._ru3[0], self._rv3[0]
                phase("k_rhs3d", lambda: (check(lib.sf_roms_rhs3d(
                    c, p(self.u), p(self.v), p(self.Huon), p(self.Hvom), p(self.Hz),
                    p(self.ru), p(self.rv), st), "sf_roms_rhs3d"), check(lib.sf_roms_stress3d(
                        c, p(self.u), p(self.v), p(self.ru), p(self.rv), p(self.sustr),
                        p(self.svstr), self.rdrag2, st), "sf_roms_stress3d")))
                phase("barotropic_loop", lambda: self._roms_loop(s, st))
                after(cs, ev_mix)
            elif ovl_rhs:
                e_flux = mark(cs)
                after(s_side, e_flux)
                phase("k_rhs3d", lambda: rhs(h(s_side)), s_side)
                after(s_loop, e_flux)
                phase("barotropic_loop", lambda: loop(h(s_loop)), s_loop)
                after(cs, mark(s_side), mark(s_loop), ev_mix)
            else:
                phase("k_rhs3d", lambda: rhs(st))
                phase("barotropic_loop", lambda: loop(st))
                after(cs, ev_mix)
            self._sync_slots(s)
            self.time2D = t2.value
            phase("k_set_depth", lambda: self.set_depth(st))
            if self.semantics == "roms":
                phase("k_step3d_uv", lambda: (check(lib.sf_roms_step3d_uv(
                    c, p(self.u), p(self.v), *[p(t) for t in self._ru3],
                    *[p(t) for t in self._rv3], p(self._slot("ubar", 1)),
                    p(self._slot("vbar", 1)), p(self._slot("ubar", 2)),
                    p(self._slot("vbar", 2)), p(self.Hz), p(self.AKv), p(self.z_r), p(self.W),
                    p(self.DU_avg1), p(self.DV_avg1), self.iic, self.ntfirst, self.lam, self.dt,
                    st), "sf_roms_step3d_uv"), check(lib.sf_lateral_uv_bc(
                        c, self.time, p(self.u), p(self.v), st), "sf_lateral_uv_bc"),
                    check(lib.sf_roms_closed_walls(c, p(self.u), p(self.v), st),
                          "sf_roms_closed_walls")))
            else:
                phase("k_step3d_uv", lambda: check(lib.sf_step3d_uv_bc(
                    c, p(self.u), p(self.v), p(self.ru), p(self.rv), p(self._slot("ubar", 1)),
                    p(self._slot("vbar", 1)), p(self._slot("ubar", 2)),
                    p(self._slot("vbar", 2)), p(self.Hz), p(self.AKv), p(self.z_r),
                    p(self.DU_avg1), p(self.DV_avg1), self.iic, self.ntfirst, self.lam, self.dt,
                    self.time, st), "sf_step3d_uv_bc"))
            if self.mixing is not None:
                if mix_ovl:
                    after(s_mix, mark(cs))
                    with torch.cuda.stream(s_mix):
                        phase("closure", self.mixing, s_mix)
                    ev_mix = mark(s_mix)
                else:
                    phase("closure", self.mixing)
            if final_omega and k == nsteps - 1:
                phase("k_omega", lambda: check(lib.sf_omega(
                    c, p(self.W), p(self.Huon), p(self.Hvom), p(self.z_w), st), "sf_omega"))
            self.iic += 1                          # CompTimes.nextTimeStep
            self.time += self.dt
            self.time2D = self.time
            if self.check_every and self.iic % self.check_every == 0:
                if ev_mix is not None:
                    cs.wait_event(ev_mix)
                self.check_state(st)
        if ev_mix is not None:   # the caller's stream sees the last mixing too
            cs.wait_event(ev_mix)
