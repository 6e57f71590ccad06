"""The reference's one-time host set-up, restated for the oracle side (TEST INFRASTRUCTURE).

The reference computes these in Python before its first step; this module restates them so
that the reference arm of the benchmark and the CPU baseline can build a basin without the
product package:

* ``weights``   nonlinear/set_weights.py:45-231   power-law barotropic averaging filter
* ``scoord``    nonlinear/set_coords.py:136-191, 364-423   S-coordinate tables (Vstretching 4)
* ``metrics``   modules/mod_grid.py:197-243        on_u, om_v, fomn
* ``lbc_lists`` modules/mod_boundary.py:103-297    boundary index lists and field maps
* ``basin``     the synthetic analytic basins the benchmark runs (tanh shelf, Gaussian
                seamounts, beta-plane Coriolis), the same recipe as the package's configs

Each routine is pinned bit for bit against the reference's own outputs in
tests/golden/setup.npz (tests/test_ref_setup.py).  Only tests/, __graft_entry__.smoke() and
bench.py's reference arm / CPU-baseline leg use this module.
"""
import numpy as np


# ---- set_weights (nonlinear/set_weights.py:45-231) ------------------------------------------
def _seq_sums(w, n):
    """Left-to-right sums of w[0:n] and of (i+1) w[i], in the reference's loop order."""
    s, m = 0.0, 0.0
    for i in range(n):
        s += w[i]
        m += (i + 1) * w[i]
    return s, m


def weights(ndtfast, size=257):
    """(nfast, weight1, weight2): shape function xi^2 (1 - xi^4) - g xi (Falpha=2, Fbeta=4,
    Fgamma=0.284, set_weights.py:37-39), scaled until its centroid is at ndtfast, shifted to
    place the centroid exactly (the reference's shift loops end at index 2, :148,:156), then
    the secondary weights and the normalisation (:165-196)."""
    a, b, g0 = 2.0, 4.0, 0.284
    nd = int(ndtfast)
    w1 = [0.0] * size
    w2 = [0.0] * size
    scale = (a + 1.0) * (a + b + 1.0) / ((a + 2.0) * (a + b + 2.0) * nd)
    gam = g0 * max(0.0, 1.0 - 10.0 / nd)
    nf = 0
    for _ in range(16):                               # set_weights.py:96-123
        nf = 0
        for i in range(2 * nd):
            x = scale * (i + 1)
            w1[i] = (x ** a) - (x ** (a + b)) - gam * x
            if w1[i] > 0.0:
                nf = i + 1
            if nf > 0 and w1[i] < 0.0:
                w1[i] = 0.0
        s, m = _seq_sums(w1, nf)
        scale = scale * m / (s * nd)
    for _ in range(nd):                               # set_weights.py:131-163
        s, m = _seq_sums(w1, nf)
        d = nd - m / s
        if d > 1.0:
            nf += 1
            for i in range(nf - 1, 1, -1):
                w1[i] = w1[i - 1]
            w1[0] = 0.0
        elif d > 0.0:
            keep = 1.0 - d
            for i in range(nf - 1, 1, -1):
                w1[i] = keep * w1[i] + d * w1[i - 1]
            w1[0] = keep * w1[0]
        elif d < -1.0:
            raise RuntimeError("centroid shift below -1: the reference fails here (:163)")
        elif d < 0.0:
            keep = 1.0 + d
            for i in range(nf - 1):
                w1[i] = keep * w1[i] - d * w1[i + 1]
            w1[nf] = keep * w1[nf]
    for j in range(nf):                               # set_weights.py:165-172
        for i in range(j):
            w2[i] += w1[j]
    s1, s2 = 0.0, 0.0
    for i in range(nf):
        s1 += w1[i]
        s2 += w2[i]
    r1, r2 = 1.0 / s1, 1.0 / s2
    for i in range(nf):
        w1[i] = r1 * w1[i]
        w2[i] = r2 * w2[i]
    return nf, np.array(w1), np.array(w2)


# ---- set_coords, Vstretching 4 (nonlinear/set_coords.py:136-191, 364-423) -------------------
def _stretch4(theta_s, theta_b, s):
    if s == 0.0:
        return 0.0
    c = (1.0 - np.cosh(theta_s * s)) / (np.cosh(theta_s) - 1.0) if theta_s > 0.0 else -s ** 2
    return (np.exp(theta_b * c) - 1.0) / (1.0 - np.exp(-theta_b)) if theta_b > 0.0 else c


def scoord(N, theta_s, theta_b):
    """(sc_r, sc_w, Cs_r, Cs_w) for Vstretching 4 (Shchepetkin 2010)."""
    ds = 1.0 / N
    sc_w = np.zeros(N + 1)
    Cs_w = np.zeros(N + 1)
    sc_r = np.zeros(N)
    Cs_r = np.zeros(N)
    sc_w[0] = Cs_w[0] = -1.0
    for k in range(1, N + 1):
        sc_w[k] = ds * (k - N)
        sc_r[k - 1] = ds * (k - N - 0.5)
        Cs_w[k] = _stretch4(theta_s, theta_b, sc_w[k])
        Cs_r[k - 1] = _stretch4(theta_s, theta_b, sc_r[k - 1])
    sc_w[N] = Cs_w[N] = 0.0
    return sc_r, sc_w, Cs_r, Cs_w


# ---- metrics (modules/mod_grid.py:197-243) --------------------------------------------------
def metrics(pm, pn, f):
    """on_u (averaged along axis 0, row 0 left 0), om_v (along axis 1, column 0 left 0) and
    fomn = f / (pm pn), as Grid.updateMetrics computes them."""
    on_u = np.zeros_like(pn)
    on_u[1:] = 2.0 / (pn[1:] + pn[:-1])
    om_v = np.zeros_like(pm)
    om_v[:, 1:] = 2.0 / (pm[:, 1:] + pm[:, :-1])
    return on_u, om_v, f * (1.0 / (pm * pn))


# ---- boundary lists (modules/mod_boundary.py:28-297) ----------------------------------------
BIT = {"CLA": (1 << 3) | 1, "CLO": 1 << 4, "GRA": 1 << 6}
CLOSED, GRADIENT, CLAMPED = 1 << 4, 1 << 6, 1 << 3


def _side_lists(codes, i0, j0, L, M):
    """buildLBC (:103-200): W column i0, E column L-1, then row i0 and row M-1 (the
    reference's third and fourth blocks), each with its destination (idx1) and source (idx2)."""
    I = L + 1
    rows = np.arange(j0, M)
    cols = np.arange(i0, L)
    blocks = [(rows * I + i0, rows * I + i0, rows * I + i0 + 1, codes[0]),
              (rows * I + L - 1, rows * I + L, rows * I + L - 1, codes[2]),
              (i0 * I + cols, i0 * I + cols, (i0 + 1) * I + cols, codes[3]),
              ((M - 1) * I + cols, M * I + cols, (M - 1) * I + cols, codes[1])]
    cat = lambda k: np.concatenate([blk[k] for blk in blocks]).astype(np.int32)
    lbc = np.concatenate([np.full(blk[0].size, blk[3], np.int32) for blk in blocks])
    return cat(0), cat(1), cat(2), lbc


def lbc_lists(L, M, spec):
    """The arrays main3d's kernels and scatters read, keyed as in oracle.Boundary.  `spec`
    maps isFsur/isUbar/isVbar/isUvel/isVvel to four keywords in the order W, S, E, N."""
    out = {}
    shp = (M + 1, L + 1)
    origin = {"zetaBC": (0, 0), "ubarBC": (1, 0), "vbarBC": (0, 1), "uvelBC": (1, 0),
              "vvelBC": (0, 1)}
    key = {"zetaBC": "isFsur", "ubarBC": "isUbar", "vbarBC": "isVbar", "uvelBC": "isUvel",
           "vvelBC": "isVvel"}
    lists = {}
    for name, (i0, j0) in origin.items():
        codes = [BIT[w.upper()] for w in spec[key[name]].split()]
        idx, i1, i2, lbc = _side_lists(codes, i0, j0, L, M)
        fidx, ftyp = np.full(shp, -1, np.int32), np.full(shp, -1, np.int32)
        fidx.reshape(-1)[i1] = i2                    # last write wins, as NumPy assigns
        ftyp.reshape(-1)[i1] = lbc
        lists[name] = (i1, i2, lbc)
        out.update({name + "_bcIdx": idx, name + "_bcIdx1": i1, name + "_bcIdx2": i2,
                    name + "_bcIdxFieldIdx2": fidx, name + "_bcIdxFieldType": ftyp,
                    name + "_LBC": lbc})
    z1, z2, zl = lists["zetaBC"]
    u1, u2, ul = lists["ubarBC"]
    v1, v2, vl = lists["vbarBC"]
    zsel = (zl & (CLOSED | GRADIENT)) != 0
    out["zetaClosedOrGradientBCIdx1"], out["zetaClosedOrGradientBCIdx2"] = z1[zsel], z2[zsel]
    out["zetaClampedBCIdx1"] = z1[(zl & CLAMPED) != 0]
    out["ubarClosedBCIdx1"], out["vbarClosedBCIdx1"] = u1[(ul & CLOSED) != 0], v1[(vl & CLOSED) != 0]
    out["ubarClampedBCIdx1"], out["vbarClampedBCIdx1"] = u1[(ul & CLAMPED) != 0], v1[(vl & CLAMPED) != 0]
    usel, vsel = (ul & GRADIENT) != 0, (vl & GRADIENT) != 0
    out["ubarGradientBCIdx1"], out["ubarGradientBCIdx2"] = u1[usel], u2[usel]
    out["vbarGradientBCIdx1"], out["vbarGradientBCIdx2"] = v1[vsel], v2[vsel]
    return out


# ---- the analytic basins ------------------------------------------------------------------
ALL_CLOSED = {k: "Clo Clo Clo Clo" for k in ("isFsur", "isUbar", "isVbar", "isUvel", "isVvel")}
BASINS = {   # Lm, Mm, N, dx, seamounts (relative x, y), dt, ndtfast
    "basin1": (512, 256, 32, 2.0e3, ((0.5, 0.6),), 240.0, 30),
    "basin4": (2048, 1024, 50, 1.0e3, ((1.0 / 3.0, 0.6), (2.0 / 3.0, 0.6)), 120.0, 40),
    "basin4q": (1024, 512, 50, 2.0e3, ((1.0 / 3.0, 0.6), (2.0 / 3.0, 0.6)), 120.0, 40),
}


def basin(name, shrink=1):
    """dict(L, M, N, h, pm, pn, on_u, om_v, fomn, sc_r, sc_w, Cs_r, Cs_w, hc, Vtransform, dt,
    ndtfast, lists) of basin `name` (shrink > 1: Lm/shrink x Mm/shrink, same recipe, dx, dt
    and ndtfast): depth 50 + 3950 x (tanh shelf across y, centred at a quarter of the
    width, width a tenth), minus 2000 m Gaussian seamounts of radius 20 km, floored at 50 m;
    f = 1e-4 + 2e-11 (y - Ly/2); uniform spacing dx; S-coordinates Vtransform 2, Vstretching
    4, theta_s 5, theta_b 0.4, hc 100 m; closed walls."""
    Lm, Mm, N, dx, mounts, dt, nd = BASINS[name]
    Lm, Mm = Lm // shrink, Mm // shrink
    L, M = Lm + 1, Mm + 1
    y = (np.arange(M + 1, dtype=np.float64)[:, None] - 0.5) * dx + np.zeros((1, L + 1))
    x = (np.arange(L + 1, dtype=np.float64)[None, :] - 0.5) * dx + np.zeros((M + 1, 1))
    Ly, Lx = Mm * dx, Lm * dx
    h = 50.0 + (4000.0 - 50.0) * (0.5 * (1.0 + np.tanh((y - 0.25 * Ly) / (0.1 * Ly))))
    for fx, fy in mounts:
        h = h - 2000.0 * np.exp(-((x - fx * Lx) ** 2 + (y - fy * Ly) ** 2) / 20.0e3 ** 2)
    h = np.maximum(h, 50.0)
    f = 1e-4 + 2e-11 * (y - 0.5 * Mm * dx)
    pm = np.full((M + 1, L + 1), 1.0 / dx)
    pn = np.full((M + 1, L + 1), 1.0 / dx)
    on_u, om_v, fomn = metrics(pm, pn, f)
    sc_r, sc_w, Cs_r, Cs_w = scoord(N, 5.0, 0.4)
    return dict(L=L, M=M, N=N, h=h, pm=pm, pn=pn, on_u=on_u, om_v=om_v, fomn=fomn, sc_r=sc_r,
                sc_w=sc_w, Cs_r=Cs_r, Cs_w=Cs_w, hc=100.0, Vtransform=2, dt=dt, ndtfast=nd,
                lists=lbc_lists(L, M, ALL_CLOSED))


def cells(name):
    Lm, Mm, N = BASINS[name][:3]
    return Lm * Mm * N

