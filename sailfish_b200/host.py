"""Host-side set-up of the time step: the reference's one-time Python routines, restated.

* ``set_weights``  -- barotropic time-averaging filter (nonlinear/set_weights.py:45-231)
* ``set_coords``   -- S-coordinate stretching tables (nonlinear/set_coords.py:10-423)
* ``update_metrics`` -- horizontal metrics (modules/mod_grid.py:197-243)
* ``Boundary``     -- lateral-boundary index lists and field maps (modules/mod_boundary.py:28-297)

They run once per grid on the host, in FP64, and are pinned bit for bit against the
reference's own outputs (tests/golden/setup.npz).  The arithmetic is NumPy float64 with the
same operand types as the reference (its arrays are CuPy float64; on the host they are NumPy
float64), so that every intermediate rounds the same way.
"""
import numpy as np

# --------------------------------------------------------------------------------------------
# set_weights (nonlinear/set_weights.py)
# --------------------------------------------------------------------------------------------
FALPHA, FBETA, FGAMMA = 2.0, 4.0, 0.284     # set_weights.py:37-39 (POWER_LAW, :41)


def set_weights(ndtfast, nweights=257):
    """Returns (nfast, weight1, weight2) for `ndtfast` barotropic steps per baroclinic step.

    Power-law shape filter F(xi) = xi^a (1 - xi^b) - g xi, centroid placed at ndtfast, then
    secondary weights for the backward-Euler free surface and normalisation
    (set_weights.py:63-196).  The reference's shift loops stop at index 2
    (``range(nfast-1, 1, -1)``, :148,:156) and that is kept.
    """
    ndtfast = int(ndtfast)
    if not 1 <= ndtfast <= (nweights - 1) // 2:
        raise ValueError("ndtfast must be in [1, %d]" % ((nweights - 1) // 2))
    w1 = np.zeros(nweights, dtype=np.float64)
    w2 = np.zeros(nweights, dtype=np.float64)
    nfast = 0
    scale = (FALPHA + 1.0) * (FALPHA + FBETA + 1.0) / ((FALPHA + 2.0) * (FALPHA + FBETA + 2.0) * ndtfast)
    gamma = FGAMMA * max(0.0, 1.0 - 10.0 / ndtfast)
    for _ in range(16):
        nfast = 0
        for i in range(2 * ndtfast):
            cff = scale * (i + 1)
            w1[i] = (cff ** FALPHA) - (cff ** (FALPHA + FBETA)) - gamma * cff
            if w1[i] > 0.0:
                nfast = i + 1
            if (nfast > 0) and (w1[i] < 0.0):
                w1[i] = 0.0
        wsum = 0.0
        shift = 0.0
        for i in range(nfast):
            wsum += w1[i]
            shift += (i + 1) * w1[i]
        scale = scale * shift / (wsum * ndtfast)

    for _ in range(ndtfast):
        wsum = 0.0
        shift = 0.0
        for i in range(nfast):
            wsum += w1[i]
            shift += (i + 1) * w1[i]
        shift = shift / wsum
        cff = ndtfast - shift
        if cff > 1.0:
            nfast += 1
            for i in range(nfast - 1, 1, -1):
                w1[i] = w1[i - 1]
            w1[0] = 0.0
        elif cff > 0.0:
            wsum = 1.0 - cff
            for i in range(nfast - 1, 1, -1):
                w1[i] = wsum * w1[i] + cff * w1[i - 1]
            w1[0] = wsum * w1[0]
        elif cff < -1.0:
            # The reference iterates `range(compTimes)` here (set_weights.py:163) and stops
            # with a TypeError; no centroid this far off has been seen for ndtfast <= 128.
            raise RuntimeError("set_weights: centroid shift < -1 (the reference fails here)")
        elif cff < 0.0:
            wsum = 1.0 + cff
            for i in range(nfast - 1):
                w1[i] = wsum * w1[i] - cff * w1[i + 1]
            w1[nfast] = wsum * w1[nfast]

    for j in range(nfast):
        cff = w1[j]
        for i in range(j):
            w2[i] += cff
    wsum = 0.0
    cff = 0.0
    for i in range(nfast):
        wsum += w1[i]
        cff += w2[i]
    wsum = 1.0 / wsum
    cff = 1.0 / cff
    for i in range(nfast):
        w1[i] = wsum * w1[i]
        w2[i] = cff * w2[i]
    return nfast, w1, w2


def roms_weights(nfast, weight1):
    """ROMS-indexed averaging weights (W1, W2) for the ROMS-form barotropic step.  set_weights
    stores ROMS's weight(1, m) at index m-1 (its loops start at iter = 1, set_weights.py:96),
    so W1[m] = weight1[m-1]; ROMS's secondary weights are weight(2, i) = sum_{j=i..nfast}
    weight(1, j), normalised over i = 1..nfast (set_weights.py:165-196 in ROMS's index
    range)."""
    W1 = np.zeros(len(weight1) + 1)
    W1[1:] = np.asarray(weight1, np.float64)
    W2 = np.zeros_like(W1)
    for i in range(1, nfast + 1):
        W2[i] = float(np.sum(W1[i:nfast + 1]))
    W2[1:nfast + 1] /= float(np.sum(W2[1:nfast + 1]))
    return W1, W2


# --------------------------------------------------------------------------------------------
# set_coords (nonlinear/set_coords.py)
# --------------------------------------------------------------------------------------------
def _cs1(theta_b, theta_s, sc):          # set_coords.py:10-34 (Song and Haidvogel 1994)
    if theta_s != 0.0:
        cff1 = 1.0 / np.sinh(theta_s)
        cff2 = 0.5 / np.tanh(theta_s * 0.5)
        w2 = 1.0 - theta_b
        w1 = theta_b
        return w2 * cff1 * np.sinh(theta_s * sc) + w1 * (cff2 * np.tanh(theta_s * (sc + 0.5)) - 0.5)
    return sc


def _cs2(theta_b, theta_s, sc):          # set_coords.py:36-82 (Shchepetkin 2005)
    Aweight, Bweight = 1.0, 1.0
    if sc == 0.0:
        return 0.0
    if theta_s > 0.0:
        Csur = (1.0 - np.cosh(theta_s * sc)) / (np.cosh(theta_s) - 1.0)
        if theta_b > 0.0:
            Cbot = np.sinh(theta_b * (sc + 1.0)) / np.sinh(theta_b) - 1.0
            Cweight = ((sc + 1.0) ** Aweight) * (1.0 + (Aweight / Bweight) * (1.0 - (sc + 1.0) ** Bweight))
            return Cweight * Csur + (1.0 - Cweight) * Cbot
        return Csur
    return sc


def _cs3(theta_b, theta_s, sc):          # set_coords.py:84-134 (Geyer)
    if sc == 0.0:
        return 0.0
    Hscale = 3.0
    Cbot = np.log(np.cosh(Hscale * (sc + 1.0) ** theta_b)) / np.log(np.cosh(Hscale)) - 1.0
    Csur = -np.log(np.cosh(Hscale * abs(sc) ** theta_s)) / np.log(np.cosh(Hscale))
    Cweight = 0.5 * (1.0 - np.tanh(Hscale * (sc + 0.5)))
    return Cweight * Cbot + (1.0 - Cweight) * Csur


def _cs4(theta_b, theta_s, sc):          # set_coords.py:136-191 (Shchepetkin 2010)
    if sc == 0.0:
        return 0.0
    if theta_s > 0.0:
        Csur = (1.0 - np.cosh(theta_s * sc)) / (np.cosh(theta_s) - 1.0)
    else:
        Csur = -sc ** 2
    if theta_b > 0.0:
        return (np.exp(theta_b * Csur) - 1.0) / (1.0 - np.exp(-theta_b))
    return Csur


_CS = {1: _cs1, 2: _cs2, 3: _cs3, 4: _cs4}


def set_coords(N, Vstretching, theta_s, theta_b):
    """S-coordinate tables (sc_r[N], sc_w[N+1], Cs_r[N], Cs_w[N+1]), set_coords.py:364-423.

    Vstretching 5 is refused, as the reference refuses it (set_coords.py:411-412)."""
    if Vstretching not in _CS:
        raise ValueError("Vstretching must be 1..4 (the reference stops on 5, set_coords.py:412)")
    N = int(N)
    sc_r = np.zeros(N)
    sc_w = np.zeros(N + 1)
    Cs_r = np.zeros(N)
    Cs_w = np.zeros(N + 1)
    sc_w[0] = -1.0
    Cs_w[0] = -1.0
    ds = 1.0 / N
    f = _CS[Vstretching]
    for k in range(1, N + 1):
        sc_w[k] = ds * (k - N)
        sc_r[k - 1] = ds * (k - N - 0.5)
        Cs_w[k] = f(theta_b, theta_s, sc_w[k])
        Cs_r[k - 1] = f(theta_b, theta_s, sc_r[k - 1])
    sc_w[N] = 0.0
    Cs_w[N] = 0.0
    return sc_r, sc_w, Cs_r, Cs_w


# --------------------------------------------------------------------------------------------
# Horizontal metrics (modules/mod_grid.py:197-243)
# --------------------------------------------------------------------------------------------
def update_metrics(pm, pn, f):
    """Metric terms of Grid.updateMetrics.  As in the reference, the 1/n and 1/m factors at
    U and V points are averaged along the first and second array axes respectively, and the
    first row of on_u/om_u and first column of om_v/on_v stay 0."""
    pm = np.asarray(pm, np.float64)
    pn = np.asarray(pn, np.float64)
    f = np.asarray(f, np.float64)
    out = {}
    out["om_r"] = 1.0 / pm
    out["on_r"] = 1.0 / pn
    out["omn"] = 1.0 / (pm * pn)
    out["fomn"] = f * out["omn"]
    om_u = np.zeros_like(pm)
    on_u = np.zeros_like(pm)
    om_u[1:, :] = 2.0 / (pm[:-1, :] + pm[1:, :])
    on_u[1:, :] = 2.0 / (pn[:-1, :] + pn[1:, :])
    om_v = np.zeros_like(pm)
    on_v = np.zeros_like(pm)
    om_v[:, 1:] = 2.0 / (pm[:, :-1] + pm[:, 1:])
    on_v[:, 1:] = 2.0 / (pn[:, :-1] + pn[:, 1:])
    out.update(om_u=om_u, on_u=on_u, om_v=om_v, on_v=on_v)
    return out


# --------------------------------------------------------------------------------------------
# Lateral boundary conditions (modules/mod_boundary.py)
# --------------------------------------------------------------------------------------------
bcNone, bcAcquire, bcChapman_explicit, bcChapman_implicit = 0, 1 << 0, 1 << 1, 1 << 2
bcClamped, bcClosed, bcFlather, bcGradient = 1 << 3, 1 << 4, 1 << 5, 1 << 6
bcMixed, bcNested, bcNudging, bcPeriodic = 1 << 7, 1 << 8, 1 << 9, 1 << 10
bcRadiation, bcReduced, bcShchepetkin = 1 << 11, 1 << 12, 1 << 13

LBC_CODES = {                             # mod_boundary.py:45-57
    "CHA": bcChapman_explicit, "CHE": bcChapman_implicit, "CLA": bcClamped + bcAcquire,
    "CLO": bcClosed, "FLA": bcFlather + bcAcquire, "GRA": bcGradient, "NES": bcNested,
    "RAD": bcRadiation, "RADNUD": bcRadiation + bcNudging + bcAcquire, "RED": bcReduced,
    "SHC": bcShchepetkin,
}
iW, iS, iE, iN = 0, 1, 2, 3


def decode_lbc(val):
    """LBC keyword -> bit set (mod_boundary.py:59-66)."""
    try:
        return LBC_CODES[val.upper()]
    except KeyError:
        raise ValueError('LBC type "%s" is not recognized' % val) from None


class BCIdx:
    """One field's boundary lists (mod_boundary.py:89-99)."""

    def __init__(self, bcIdx, bcIdx1, bcIdx2, bcIdxFieldIdx2, bcIdxFieldType, LBC):
        self.bcIdx, self.bcIdx1, self.bcIdx2 = bcIdx, bcIdx1, bcIdx2
        self.bcIdxFieldIdx2, self.bcIdxFieldType, self.LBC = bcIdxFieldIdx2, bcIdxFieldType, LBC


def build_lbc(val, i0, j0, L, M):
    """Boundary.buildLBC (mod_boundary.py:103-200).  Blocks in the order W, E, "N", "S": the
    third block is the row i0 and the fourth the row M (the reference labels them N and S and
    indexes the third with i0 as a row); field maps are written with NumPy's last-wins rule
    for repeated nodes."""
    shp = (M + 1, L + 1)
    bcW, bcE, bcN, bcS = (decode_lbc(val[k]) for k in (iW, iE, iN, iS))
    iR = np.arange(i0, L)
    jR = np.arange(j0, M)
    idx, idx1, idx2, lbc = [], [], [], []
    for a, a1, a2, code, n in (
            ((jR, [i0]), (jR, [i0]), (jR, [i0 + 1]), bcW, M - j0),
            ((jR, [L - 1]), (jR, [L]), (jR, [L - 1]), bcE, M - j0),
            (([i0], iR), ([i0], iR), ([i0 + 1], iR), bcN, L - i0),
            (([M - 1], iR), ([M], iR), ([M - 1], iR), bcS, L - i0)):
        idx += np.ravel_multi_index((np.asarray(a[0]), np.asarray(a[1])), shp).tolist()
        idx1 += np.ravel_multi_index((np.asarray(a1[0]), np.asarray(a1[1])), shp).tolist()
        idx2 += np.ravel_multi_index((np.asarray(a2[0]), np.asarray(a2[1])), shp).tolist()
        lbc += [code] * n
    bcIdx = np.array(idx, dtype=np.int32)
    bcIdx1 = np.array(idx1, dtype=np.int32)
    bcIdx2 = np.array(idx2, dtype=np.int32)
    LBC = np.array(lbc, dtype=np.int32)
    fidx2 = -np.ones(shp, np.int32)
    ftype = -np.ones(shp, np.int32)
    fidx2.ravel()[bcIdx1] = bcIdx2
    ftype.ravel()[bcIdx1] = LBC
    return BCIdx(bcIdx, bcIdx1, bcIdx2, fidx2, ftype, LBC)


def _local_bc_idx(bc, flat):
    """Boundary.getLocalBCIdx (mod_boundary.py:202-234): position of `flat` in bc.bcIdx."""
    hits = np.nonzero(bc.bcIdx == flat)[0]
    if hits.size == 0:
        raise ValueError("Index %i not in the list" % flat)
    return int(hits[-1])


class Boundary:
    """Boundary index lists for the five fields (mod_boundary.py:237-297).

    `lbc` maps 'isFsur', 'isUbar', 'isVbar', 'isUvel', 'isVvel' to four keywords in the order
    W, S, E, N (the order of `LBC(...) ==` lines in the reference's input file)."""

    DEFAULT = {"isFsur": "Clo Clo Clo Clo", "isUbar": "Cla Clo Clo Clo", "isVbar": "Clo Clo Clo Clo",
               "isUvel": "Cla Clo Clo Clo", "isVvel": "Cla Clo Clo Clo"}   # utility/test.in:185-189

    def __init__(self, L, M, lbc=None):
        lbc = dict(self.DEFAULT, **(lbc or {}))
        sp = lambda k: lbc[k].split() if isinstance(lbc[k], str) else list(lbc[k])
        self.zetaBC = build_lbc(sp("isFsur"), 0, 0, L, M)
        self.ubarBC = build_lbc(sp("isUbar"), 1, 0, L, M)
        self.vbarBC = build_lbc(sp("isVbar"), 0, 1, L, M)
        self.uvelBC = build_lbc(sp("isUvel"), 1, 0, L, M)
        self.vvelBC = build_lbc(sp("isVvel"), 0, 1, L, M)
        for vb in (self.ubarBC, self.vbarBC):
            for k in range(vb.bcIdx.size):
                if (vb.LBC[k] & bcFlather) or (vb.LBC[k] & bcShchepetkin):
                    self.zetaBC.LBC[_local_bc_idx(self.zetaBC, vb.bcIdx[k])] |= bcAcquire
        z, u, v = self.zetaBC, self.ubarBC, self.vbarBC
        sel = ((z.LBC & bcClosed) | (z.LBC & bcGradient)) != 0
        self.zetaClosedOrGradientBCIdx1 = z.bcIdx1[sel]
        self.zetaClosedOrGradientBCIdx2 = z.bcIdx2[sel]
        self.zetaClampedBCIdx1 = z.bcIdx1[(z.LBC & bcClamped) != 0]
        self.ubarClosedBCIdx1 = u.bcIdx1[(u.LBC & bcClosed) != 0]
        self.vbarClosedBCIdx1 = v.bcIdx1[(v.LBC & bcClosed) != 0]
        self.ubarClampedBCIdx1 = u.bcIdx1[(u.LBC & bcClamped) != 0]
        self.vbarClampedBCIdx1 = v.bcIdx1[(v.LBC & bcClamped) != 0]
        sel = (u.LBC & bcGradient) != 0
        self.ubarGradientBCIdx1, self.ubarGradientBCIdx2 = u.bcIdx1[sel], u.bcIdx2[sel]
        sel = (v.LBC & bcGradient) != 0
        self.vbarGradientBCIdx1, self.vbarGradientBCIdx2 = v.bcIdx1[sel], v.bcIdx2[sel]
