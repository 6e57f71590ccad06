"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run in a container that has the reference checkout (``$SAILFISH_REFERENCE``, default: a
``reference`` directory beside the repository).  Nothing at test time reads the reference: the tests only load the
``.npz`` files written here.

How the reference is run on the CPU:
  * its CUDA kernel files are host-compiled by oracle/build_ref.py into oracle/_ref;
  * its Python orchestration (utility/io_utils.py, modules/mod_grid.py, mod_boundary.py,
    mod_comptimes.py, mod_ocean.py, mod_operators.py, nonlinear/set_coords.py,
    set_weights.py, step2d.py, rhs.py, main3d.py) is imported unmodified, with
    tests/golden/cupy_shim standing in for ``cupy`` (NumPy arrays with zero guards, and
    RawModule kernels dispatched to oracle/_ref).

Fixtures:
  setup.npz     set_weights (nfast, weight1, weight2) for several NDTFAST; set_coords
                (sc_r, sc_w, Cs_r, Cs_w) for Vstretching 1-4; Boundary index arrays and
                field maps (modules/mod_boundary.py:103-297); grid metrics
                (modules/mod_grid.py:197-243).
  kernels.npz   each reference kernel launched once, as the reference launches it, on seeded
                inputs (inputs and outputs stored).
  main3d_*.npz  the reference's main3d (nonlinear/main3d.py:25-326) run for a few baroclinic
                steps from a seeded initial state: initial state and final state.
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.abspath(os.path.join(HERE, "..", ".."))
REF = os.environ.get("SAILFISH_REFERENCE", os.path.join(os.path.dirname(REPO), "reference"))

sys.path[:0] = [os.path.join(HERE, "cupy_shim")] + [os.path.join(REF, d) for d in
                                                     ("modules", "utility", "nonlinear", "functionals")]
sys.path.insert(0, os.path.join(REPO, "oracle"))
import build_ref  # noqa: E402

build_ref.build()

import cupy as cp  # noqa: E402  (the shim)
import io_utils  # noqa: E402
import mod_grid  # noqa: E402
import mod_boundary  # noqa: E402
import mod_comptimes  # noqa: E402
import mod_ocean  # noqa: E402
import set_weights  # noqa: E402
from set_coords import set_coords  # noqa: E402
import ana_grid  # noqa: E402
import mod_operators  # noqa: E402
import step2d as ref_step2d  # noqa: E402
import rhs as ref_rhs  # noqa: E402
import main3d as ref_main3d  # noqa: E402

VARINFO = io_utils.VarInfoList(path=os.path.join(REF, "modules"))


def make_input(**over):
    """The reference's utility/test.in with `KEY == value` overrides appended (the parser
    keeps the last assignment of a key, utility/io_utils.py:82-94)."""
    with open(os.path.join(REF, "utility", "test.in")) as f:
        text = f.read()
    text += "\n" + "\n".join("%s == %s" % (k, v) for k, v in over.items()) + "\n"
    fd, path = tempfile.mkstemp(suffix=".in")
    with os.fdopen(fd, "w") as f:
        f.write(text)
    inp = io_utils.Input(path, VARINFO)
    os.unlink(path)
    return inp


def build_case(Lm, Mm, N, ndtfast=30, dt=30.0, vtransform=2, vstretching=4, theta_s=5.0,
               theta_b=0.4, tcline=100.0, grid="basin", f0=1e-4, beta=2e-11, seed=0):
    inp = make_input(Lm=Lm, Mm=Mm, N=N, NDTFAST=ndtfast, DT=dt, Vtransform=vtransform,
                     Vstretching=vstretching, THETA_S=theta_s, THETA_B=theta_b, TCLINE=tcline)
    GRID = mod_grid.Grid(inp)
    BOUNDARY = mod_boundary.Boundary(inp, GRID)
    compTimes = mod_comptimes.CompTimes(inp)
    OCEAN = mod_ocean.T_OCEAN(inp, GRID)
    if grid == "basin":
        ana_grid.ana_grid("Basin", GRID)         # square grids only (functionals/anaBASE.py:17)
        y = GRID.yr.T if GRID.yr.shape != GRID.f.shape else GRID.yr
    else:
        # Non-square analytic grid set the way functionals/anaBASE.py sets the Basin one.
        # Large cells and a shallow basin: the reference's barotropic scheme amplifies
        # perturbations at a rate that grows with the gravity-wave Courant number, so the
        # fixtures use a small one to stay finite over their few steps.
        dx, dy = 250.0e3, 200.0e3
        GRID.pm[:, :] = 1.0 / dx
        GRID.pn[:, :] = 1.0 / dy
        jj, ii = np.meshgrid(np.arange(GRID.M + 1), np.arange(GRID.L + 1), indexing="ij")
        y = (jj - 0.5) * dy
        GRID.h[:, :] = 30.0 + 10.0 * (1.0 + np.tanh((jj - GRID.M / 2.0) / 2.0)) + 0.5 * ii
        GRID.hmin, GRID.hmax = GRID.h.min(), GRID.h.max()
    GRID.f[:, :] = f0 + beta * (y - y.mean())
    GRID.updateMetrics()
    set_coords(GRID)
    set_weights.set_weights(compTimes)
    mod_operators.initModule(GRID)
    mod_operators.set_depth(mod_operators.grsz, mod_operators.bksz,
                            (GRID.Vtransform, OCEAN.Zt_avg1, GRID.z_w, GRID.z_r, GRID.h, GRID.hc,
                             GRID.Hz, GRID.sc_r, GRID.sc_w, GRID.Cs_r, GRID.Cs_w))
    OCEAN.AKv[:, :, :] = 2.0e-3 + 8.0e-3 * np.exp(GRID.z_w / 150)   # tmp/testProgram.py:75
    return GRID, BOUNDARY, compTimes, OCEAN


def grid_arrays(GRID):
    return {k: np.array(getattr(GRID, k)) for k in
            ("h", "f", "pm", "pn", "on_u", "om_v", "fomn", "om_u", "on_v", "omn",
             "sc_r", "sc_w", "Cs_r", "Cs_w", "z_w", "z_r", "Hz")} | {"hc": GRID.hc}


def boundary_arrays(B, prefix=""):
    out = {}
    for name in ("zetaBC", "ubarBC", "vbarBC", "uvelBC", "vvelBC"):
        bc = getattr(B, name)
        for f in ("bcIdx", "bcIdx1", "bcIdx2", "bcIdxFieldIdx2", "bcIdxFieldType", "LBC"):
            out["%s%s_%s" % (prefix, name, f)] = np.array(getattr(bc, f))
    for f in ("zetaClosedOrGradientBCIdx1", "zetaClosedOrGradientBCIdx2", "zetaClampedBCIdx1",
              "ubarClosedBCIdx1", "vbarClosedBCIdx1", "ubarClampedBCIdx1", "vbarClampedBCIdx1",
              "ubarGradientBCIdx1", "ubarGradientBCIdx2", "vbarGradientBCIdx1", "vbarGradientBCIdx2"):
        out[prefix + f] = np.array(getattr(B, f))
    return out


# ----------------------------------------------------------------------------------------
def gen_setup():
    out = {}
    for nd in (10, 20, 30, 40, 60):
        inp = make_input(NDTFAST=nd)
        ct = mod_comptimes.CompTimes(inp)
        set_weights.set_weights(ct)
        out["weights_%d_nfast" % nd] = np.array(ct.nfast)
        out["weights_%d_w1" % nd] = np.array(ct.weight1)
        out["weights_%d_w2" % nd] = np.array(ct.weight2)
    for vs, ts, tb in ((1, 5.0, 0.4), (1, 0.0, 0.0), (2, 5.0, 0.4), (2, 3.0, 0.0), (3, 0.65, 0.58),
                       (4, 5.0, 0.4), (4, 0.0, 0.0), (4, 7.0, 2.0)):
        inp = make_input(Lm=12, Mm=12, N=7, Vstretching=vs, THETA_S=ts, THETA_B=tb)
        G = mod_grid.Grid(inp)
        ana_grid.ana_grid("Basin", G)
        set_coords(G)
        key = "coords_v%d_%g_%g" % (vs, ts, tb)
        for f in ("sc_r", "sc_w", "Cs_r", "Cs_w"):
            out[key + "_" + f] = np.array(getattr(G, f))
    for Lm, Mm in ((12, 12), (16, 10), (9, 14)):
        inp = make_input(Lm=Lm, Mm=Mm, N=4)
        G = mod_grid.Grid(inp)
        B = mod_boundary.Boundary(inp, G)
        out.update(boundary_arrays(B, prefix="bnd_%dx%d_" % (Lm, Mm)))
    GRID, *_ = build_case(16, 10, 5, grid="nonsquare")
    out.update({"metrics_16x10_" + k: v for k, v in grid_arrays(GRID).items()})
    np.savez_compressed(os.path.join(HERE, "setup.npz"), **out)


# ----------------------------------------------------------------------------------------
def gen_kernels():
    """Each reference kernel once, with the reference's own launch geometry."""
    rng = np.random.default_rng(1234)
    GRID, B, ct, OCEAN = build_case(16, 10, 5, grid="nonsquare", vtransform=2)
    N, M, L = GRID.N, GRID.M, GRID.L
    sh2, sh3, sh3w = (M + 1, L + 1), GRID.shape3D, GRID.shape3DW
    grsz, bksz, GPUMUL = mod_operators.grsz, mod_operators.bksz, 2
    out = {"N": N, "M": M, "L": L}
    out.update({"grid_" + k: v for k, v in grid_arrays(GRID).items()})
    out.update(boundary_arrays(B, prefix="bnd_"))

    def rnd(shape, scale=1.0, offset=0.0):
        a = cp.zeros(shape)
        a[...] = offset + scale * rng.standard_normal(shape)
        return a

    def slot3(shape, scale, offset=0.0):
        """A (3, *shape) parent like modules/mod_ocean.py:65-71; returns parent, slot-2 view."""
        p = cp.zeros((3,) + tuple(shape))
        p[...] = offset + scale * rng.standard_normal(p.shape)
        return p, p[2].ravel()

    def save(prefix, **arrs):
        for k, v in arrs.items():
            out[prefix + "_" + k] = np.array(v)

    # --- set_depth, both transforms (nonlinear/step3D_uv.kernels.cpp:225-291)
    for vt in (1, 2):
        Zt = rnd(sh2, 0.3).ravel()
        z_w, z_r, Hz = cp.zeros(sh3w), cp.zeros(sh3), cp.zeros(sh3)
        save("set_depth%d_in" % vt, Zt=Zt)
        mod_operators.set_depth(grsz, bksz, (vt, Zt, z_w, z_r, GRID.h, GRID.hc, Hz,
                                             GRID.sc_r, GRID.sc_w, GRID.Cs_r, GRID.Cs_w))
        save("set_depth%d_out" % vt, z_w=z_w, z_r=z_r, Hz=Hz)
    z_w, z_r, Hz = cp.zeros(sh3w), cp.zeros(sh3), cp.zeros(sh3)
    Zt = rnd(sh2, 0.3).ravel()
    mod_operators.set_depth(grsz, bksz, (2, Zt, z_w, z_r, GRID.h, GRID.hc, Hz,
                                         GRID.sc_r, GRID.sc_w, GRID.Cs_r, GRID.Cs_w))
    save("geom", z_w=z_w, z_r=z_r, Hz=Hz)

    # --- set_maxflux + omega (:372-405, :62-165)
    up, u = slot3(sh3w, 0.1)
    vp, v = slot3(sh3w, 0.1)
    Huon, Hvom, W = rnd(sh3w, 1.0), rnd(sh3w, 1.0), rnd(sh3w, 1.0)
    BC = B.zetaBC.bcIdxFieldIdx2.ravel()
    save("maxflux_in", u_parent=up, v_parent=vp, Huon=Huon, Hvom=Hvom, W=W)
    mod_operators.set_maxflux(grsz, bksz, (u, v, Huon, Hvom, Hz))
    save("maxflux_out", Huon=Huon, Hvom=Hvom)
    mod_operators.omega(grsz, bksz, (W, u, v, Huon.ravel(), Hvom.ravel(), z_w, BC))
    save("omega_out", W=W)

    # --- rhs3d (nonlinear/rhs.py:16-93 -> rhs_kernels.cpp)
    rup, ru = slot3(sh3w, 1.0)
    rvp, rv = slot3(sh3w, 1.0)
    save("rhs3d_in", ru_parent=rup, rv_parent=rvp)
    OCEAN.u, OCEAN.v, OCEAN.ru, OCEAN.rv = up, vp, rup, rvp
    OCEAN.u_t2, OCEAN.v_t2, OCEAN.ru_t2, OCEAN.rv_t2 = u, v, ru, rv
    OCEAN.Huon, OCEAN.Hvom, OCEAN.W = Huon, Hvom, W
    GRID.Hz[...] = Hz
    cp.launch_log.clear()
    ref_rhs.rhs3d(GRID, OCEAN, B)
    save("rhs3d_out", ru_parent=rup, rv_parent=rvp)
    out["rhs3d_launches"] = np.array([[n for (_, _, n) in cp.launch_log]])

    # --- step3d_UV + setLateralUVBCs (:646-707, :314-368)
    AKv = rnd(sh3w, 1e-3, 5e-3)
    AKv[...] = np.abs(AKv)
    DU, DV = rnd(sh2, 50.0).ravel(), rnd(sh2, 50.0).ravel()
    ub1, vb1, ub2, vb2 = (rnd(sh2, 0.1).ravel() for _ in range(4))
    tmpU, tmpV = cp.zeros(u.shape), cp.zeros(v.shape)
    tmpU[:] = u
    tmpV[:] = v
    eqSD, eqD, eqRHS = cp.zeros(sh3w), cp.zeros(sh3w), cp.zeros(sh3w)
    mod_operators.setVerticalVelEq((1,), (1,), (eqSD, eqD, eqRHS))
    save("step3d_in", AKv=AKv, DU_avg1=DU, DV_avg1=DV, ubar_t1=ub1, vbar_t1=vb1, ubar_t2=ub2,
         vbar_t2=vb2, u_parent=up, v_parent=vp)
    for iic in (0, 1, 5):
        up2, vp2 = up.copy(), vp.copy()
        uu, vv = cp.zeros(up.shape), cp.zeros(vp.shape)
        uu[...] = up2
        vv[...] = vp2
        b1, c1, b2, c2 = (cp.zeros(sh2).ravel() for _ in range(4))
        b1[:] = ub1
        c1[:] = vb1
        b2[:] = ub2
        c2[:] = vb2
        mod_operators.step3d_UV((grsz[0] * GPUMUL,), (bksz[0] // GPUMUL,),
                                (uu[2].ravel(), vv[2].ravel(), ru, rv, b1, c1, b2, c2, Hz, AKv, z_r,
                                 DU, DV, tmpU, tmpV, GRID.h, iic, 0, 1.0, 1e-5, 240.0))
        save("step3d_out_iic%d" % iic, u_parent=uu, v_parent=vv, ubar_t1=b1, vbar_t1=c1,
             ubar_t2=b2, vbar_t2=c2)
    uu, vv = cp.zeros(up.shape), cp.zeros(vp.shape)
    uu[...] = up
    vv[...] = vp
    mod_operators.setLateralUVBCs((grsz[0],), (bksz[0],),
                                  (1234.5, uu[2].ravel(), vv[2].ravel(), B.uvelBC.bcIdxFieldIdx2,
                                   B.vvelBC.bcIdxFieldIdx2, B.uvelBC.bcIdxFieldType,
                                   B.vvelBC.bcIdxFieldType))
    save("lateral_out", u_parent=uu, v_parent=vv)

    # --- set_zeta (:294-310)
    z1, z2 = rnd(sh2, 0.1).ravel(), rnd(sh2, 0.1).ravel()
    Zt = rnd(sh2, 0.1).ravel()
    save("set_zeta_in", zeta1=z1, zeta2=z2, Zt=Zt)
    mod_operators.set_zeta(grsz, bksz, (z1, z2, Zt))
    save("set_zeta_out", zeta1=z1, zeta2=z2)

    # --- 2D predictor / corrector through the reference's own step2d.py
    for name in ("zeta", "ubar", "vbar", "rzeta", "rubar", "rvbar"):
        par = getattr(OCEAN, name)
        par[...] = (0.2 if name == "zeta" else 0.05) * rng.standard_normal(par.shape)
        if name.startswith("r"):
            par[...] *= 1e-3
    OCEAN.Zt_avg1[:] = 0.1 * rng.standard_normal(OCEAN.Zt_avg1.shape)
    OCEAN.DU_avg1[:] = 10.0 * rng.standard_normal(OCEAN.DU_avg1.shape)
    OCEAN.DV_avg1[:] = 10.0 * rng.standard_normal(OCEAN.DV_avg1.shape)
    ct.iif, ct.time2D = 3, 777.0
    st = lambda: {n: np.array(getattr(OCEAN, n)) for n in
                  ("zeta", "ubar", "vbar", "rzeta", "rubar", "rvbar", "Zt_avg1", "DU_avg1", "DV_avg1")}
    save("step2d_in", **st())
    ref_step2d.step2dPredictor(ct, GRID, OCEAN, B)
    save("step2d_pred_out", **st())
    ref_step2d.step2dCorrector(ct, GRID, OCEAN, B)
    save("step2d_corr_out", **st())
    out["step2d_weights_w1"] = np.array(ct.weight1)
    out["step2d_weights_w2"] = np.array(ct.weight2)
    out["step2d_dtfast"] = np.array(ct.dtfast)
    np.savez_compressed(os.path.join(HERE, "kernels.npz"), **out)


# ----------------------------------------------------------------------------------------
def gen_main3d(tag, nsteps, **case):
    rng = np.random.default_rng(99)
    GRID, B, ct, OCEAN = build_case(**case)
    N, M, L = GRID.N, GRID.M, GRID.L
    jj, ii = np.meshgrid(np.arange(M + 1), np.arange(L + 1), indexing="ij")
    bump = 0.05 * np.exp(-(((ii - L / 2.0) / (L / 5.0)) ** 2 + ((jj - M / 2.0) / (M / 5.0)) ** 2))
    OCEAN.Zt_avg1[:] = bump.ravel()
    OCEAN.u[2][...] = 0.01 * rng.standard_normal(OCEAN.u[2].shape)
    OCEAN.v[2][...] = 0.01 * rng.standard_normal(OCEAN.v[2].shape)
    names = ("zeta", "ubar", "vbar", "rzeta", "rubar", "rvbar", "u", "v", "ru", "rv", "W",
             "Huon", "Hvom", "Zt_avg1", "DU_avg1", "DV_avg1", "AKv")
    init = {n: np.array(getattr(OCEAN, n)) for n in names}
    init.update({"grid_" + k: v for k, v in grid_arrays(GRID).items()})
    init.update(boundary_arrays(B, prefix="bnd_"))
    init.update({"N": N, "M": M, "L": L, "nfast": ct.nfast, "w1": np.array(ct.weight1),
                 "w2": np.array(ct.weight2), "dt": ct.dt, "ndtfast": ct.ndtfast,
                 "Vtransform": GRID.Vtransform, "AK": OCEAN.AK, "nsteps": nsteps})
    ct.ntend = nsteps - 1               # main3d runs while iic < ntend + 1 (mod_comptimes.py:69-71)
    ref_main3d.main3d(ct, GRID, OCEAN, B)
    fin = {n: np.array(getattr(OCEAN, n)) for n in names}
    for n in ("z_w", "z_r", "Hz"):
        fin[n] = np.array(getattr(GRID, n))
    slot = lambda view, parent: int(round((view.ctypes.data - parent.ctypes.data) / view.nbytes))
    for n in ("zeta", "ubar", "vbar", "rzeta", "rubar", "rvbar"):
        par = getattr(OCEAN, n)
        fin["slots_" + n] = np.array([slot(getattr(OCEAN, "%s_t%d" % (n, t)), par) for t in (0, 1, 2)])
    fin["time"], fin["time2D"], fin["iic"] = ct.time, ct.time2D, ct.iic
    np.savez_compressed(os.path.join(HERE, "main3d_%s.npz" % tag),
                        **{"in_" + k: v for k, v in init.items()},
                        **{"out_" + k: v for k, v in fin.items()})


if __name__ == "__main__":
    gen_setup()
    gen_kernels()
    gen_main3d("square", 3, Lm=12, Mm=12, N=6, ndtfast=30, dt=30.0, grid="basin")
    # On non-square grids computeMomentumPred's guard (mod_cppkernels.cpp:162 tests the flat
    # index against szJ) leaves interior ubar nodes holding the mis-bound corrector's
    # (modules/mod_operators.py:146) unscaled increments, and the reference's state grows by
    # orders of magnitude per barotropic substep; these cases therefore run one baroclinic
    # step with few substeps so that every value stays finite.
    gen_main3d("nonsquare", 1, Lm=16, Mm=10, N=5, ndtfast=4, dt=60.0, grid="nonsquare",
               vtransform=2, tcline=20.0)
    gen_main3d("vt1", 1, Lm=9, Mm=14, N=7, ndtfast=4, dt=30.0, grid="nonsquare",
               vtransform=1, vstretching=1, theta_s=3.0, theta_b=0.0, tcline=10.0)
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))
