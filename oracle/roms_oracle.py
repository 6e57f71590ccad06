"""ROMS-form barotropic step, restated in NumPy FP64 (TEST INFRASTRUCTURE: the oracle).

The reference's runnable 2D kernels (modules/mod_cppkernels.cpp) carry no forcing, reversed
signs and a mis-bound corrector; its ROMS transcription of the full step
(obsolete/step2d_LF_AM3.h.py) and of the bottom stress (nonlinear/set_vbc.py) do not parse.
The benchmark configurations need that physics (wind stress, quadratic bottom drag,
Coriolis), so the package has a second, ROMS-form barotropic step; this module restates it
from the pseudo-code, for closed rectangular basins (no masks, no wet/dry, no open
boundaries), vectorised over the grid:

* total depth and face fluxes DUon = ubar (D_i + D_i-1)/2 on_u, DVom likewise (:690-745);
* fast-time averages accumulated in the predictor from the previous corrector's fields:
  Zt_avg1 += W1[iif-1] zeta, DU_avg1 += W1[iif-1] DUon, DU_avg2 += (8/12 W2[iif]
  - 1/12 W2[iif+1]) DUon, reset at iif = 1 with DU_avg2 = -1/12 W2[2] DUon; in the corrector
  DU_avg2 += 5/12 W2[iif] DUon (W2[1] at iif = 1) (:778-846); W1, W2 are indexed as ROMS
  indexes weight(1:2, 0:256) (roms_weights); the predictor of substep nfast+1 only
  accumulates (:923-926);
* free surface: rhs_zeta = (DUon_i - DUon_i+1) + (DVom_j - DVom_j+1); predictor
  zeta_new = zeta(kstp) + pm pn cff1 rhs_zeta with cff1 = dtfast at the first substep of a
  loop (forward Euler, kstp = n) and 2 dtfast after (leapfrog, kstp = n-1); corrector AM3
  zeta_new = zeta(n) + pm pn dtfast (5/12 rhs + 8/12 rzeta(n) - 1/12 rzeta(n-1)) (backward
  Euler at the first substep); the pressure-gradient surface zwrk = 0.5 (zeta(kstp) +
  zeta_new) first, 0.68 zeta(n) + 0.16 (zeta(n-1) + zeta_new) in the predictor, 0.6 zeta_new +
  0.4 zeta(n+1*) in the corrector (:933-1020); zero-gradient ring (closed walls);
* momentum right-hand side at U/V faces: pressure gradient 0.5 g on_u ((h_i-1 + h_i)
  (zwrk_i-1 - zwrk_i) + (zwrk_i-1^2 - zwrk_i^2)) (:1120-1160); Coriolis from
  UFx = 0.5 Drhs fomn (vbar_j + vbar_j+1) at rho points, + (UFx_i + UFx_i-1)/2 for ubar and
  - (VFe_j + VFe_j-1)/2 for vbar (:1503-1530); surface stress + sustr om_u on_u (:2598-2612);
  quadratic bottom drag - rdrag2 ubar sqrt(ubar^2 + v_u^2) om_u on_u with v_u the four-point
  average of vbar at the U face (set_vbc.py:16-41, step2d_LF_AM3.h.py:2242-2262);
* momentum step (:2640-2760): ubar_new = (ubar(kstp) (Dstp_i + Dstp_i-1) + cff cff1 rhs) /
  (Dnew_i + Dnew_i-1), cff = (pm_i + pm_i-1)(pn_i + pn_i-1), cff1 = dtfast/2 (first),
  dtfast (leapfrog predictor), and in the corrector dtfast/2 (5/12 rhs + 8/12 rubar(n)
  - 1/12 rubar(n-1)); normal velocities on the walls are 0.

Index conventions follow the reference's arrays: (J, I) = (M+1, L+1) rho grid, ubar(j, i) on the
west face of rho (j, i), vbar(j, i) on its south face; interior rho 1..I-2 x 1..J-2, U faces
i = 2..I-2 (walls at i = 1 and I-1), V faces j = 2..J-2 (walls at j = 1 and J-1).

Time levels: each field has slots n-1, n and a scratch for the predicted n+1*; the corrector
writes n+1 over n-1, then n-1 <- n and n <- n+1 (a swap of the two slots).
"""
import numpy as np

G_GRAV = 10.0      # modules/mod_constants.py:26


def roms_weights(nfast, w1):
    """ROMS-indexed (W1, W2) from the primary weights w1 of set_weights: the reference's array
    holds ROMS weight(1, m) at index m-1 (set_weights.py:96-104 fills it from iter = 1), so
    W1[m] = w1[m-1] (W1[0] = 0); W2[i] = sum_{j=i..nfast} W1[j] (ROMS's secondary weights,
    set_weights.py:165-172 in ROMS's index range), normalised to sum 1 over i = 1..nfast."""
    W1 = np.zeros(len(w1) + 1)
    W1[1:] = np.asarray(w1, np.float64)
    W2 = np.zeros_like(W1)
    for i in range(1, nfast + 1):
        W2[i] = float(np.sum(W1[i:nfast + 1]))
    W2[1:nfast + 1] /= float(np.sum(W2[1:nfast + 1]))
    return W1, W2


class State:
    """Barotropic state of one basin (FP64 host arrays, shape (J, I))."""

    def __init__(self, J, I):
        z = lambda: np.zeros((J, I))
        self.zeta = [z(), z()]          # [n-1, n]
        self.ubar = [z(), z()]
        self.vbar = [z(), z()]
        self.rzeta = [z(), z()]
        self.rubar = [z(), z()]
        self.rvbar = [z(), z()]
        self.zeta_p, self.ubar_p, self.vbar_p = z(), z(), z()   # predicted n+1*
        self.Zt_avg1, self.DU_avg1, self.DV_avg1, self.DU_avg2, self.DV_avg2 = z(), z(), z(), z(), z()


def _fluxes(g, zeta, ubar, vbar):
    D = zeta + g["h"]
    DU = np.zeros_like(D)
    DV = np.zeros_like(D)
    DU[:, 1:] = ubar[:, 1:] * (0.5 * (D[:, 1:] + D[:, :-1])) * g["on_u"][:, 1:]
    DV[1:, :] = vbar[1:, :] * (0.5 * (D[1:, :] + D[:-1, :])) * g["om_v"][1:, :]
    return D, DU, DV


def _rhs_zeta(DU, DV):
    r = np.zeros_like(DU)
    r[1:-1, 1:-1] = ((DU[1:-1, 1:-1] - DU[1:-1, 2:]) + (DV[1:-1, 1:-1] - DV[2:, 1:-1]))
    return r


def _ring(z):
    """Zero-gradient free surface on the boundary ring (closed walls)."""
    z[0, :] = z[1, :]
    z[-1, :] = z[-2, :]
    z[:, 0] = z[:, 1]
    z[:, -1] = z[:, -2]


def _rhs_uv(g, zwrk, D, ubar, vbar, sustr, svstr, rdrag2):
    """rhs_ubar, rhs_vbar on the interior faces (zero elsewhere)."""
    h, fomn = g["h"], g["fomn"]
    J, I = h.shape
    ru = np.zeros_like(h)
    rv = np.zeros_like(h)
    cff1 = 0.5 * G_GRAV
    gz, gz2 = zwrk, zwrk * zwrk
    # U faces i = 2..I-2, rows j = 1..J-2
    sl_j, sl_i = slice(1, J - 1), slice(2, I - 1)
    sl_im = slice(1, I - 2)
    pg = cff1 * g["on_u"][sl_j, sl_i] * ((h[sl_j, sl_im] + h[sl_j, sl_i]) * (gz[sl_j, sl_im] - gz[sl_j, sl_i])
                                         + (gz2[sl_j, sl_im] - gz2[sl_j, sl_i]))
    UFx = 0.5 * D * fomn * np.concatenate([vbar[:-1] + vbar[1:], np.zeros((1, I))], axis=0)
    cor = 0.5 * (UFx[sl_j, sl_i] + UFx[sl_j, sl_im])
    area_u = 4.0 / ((g["pm"][sl_j, sl_i] + g["pm"][sl_j, sl_im]) * (g["pn"][sl_j, sl_i] + g["pn"][sl_j, sl_im]))
    v4 = 0.25 * (vbar[sl_j, sl_i] + vbar[2:J, sl_i] + vbar[sl_j, sl_im] + vbar[2:J, sl_im])
    ub = ubar[sl_j, sl_i]
    bustr = rdrag2 * ub * np.sqrt(ub * ub + v4 * v4)
    ru[sl_j, sl_i] = pg + cor + (sustr[sl_j, sl_i] - bustr) * area_u
    # V faces j = 2..J-2, columns i = 1..I-2
    sv_j, sv_i = slice(2, J - 1), slice(1, I - 1)
    sv_jm = slice(1, J - 2)
    pgv = cff1 * g["om_v"][sv_j, sv_i] * ((h[sv_jm, sv_i] + h[sv_j, sv_i]) * (gz[sv_jm, sv_i] - gz[sv_j, sv_i])
                                          + (gz2[sv_jm, sv_i] - gz2[sv_j, sv_i]))
    VFe = 0.5 * D * fomn * np.concatenate([ubar[:, :-1] + ubar[:, 1:], np.zeros((J, 1))], axis=1)
    corv = -0.5 * (VFe[sv_j, sv_i] + VFe[sv_jm, sv_i])
    area_v = 4.0 / ((g["pm"][sv_j, sv_i] + g["pm"][sv_jm, sv_i]) * (g["pn"][sv_j, sv_i] + g["pn"][sv_jm, sv_i]))
    u4 = 0.25 * (ubar[sv_j, sv_i] + ubar[sv_j, 2:I] + ubar[sv_jm, sv_i] + ubar[sv_jm, 2:I])
    vb = vbar[sv_j, sv_i]
    bvstr = rdrag2 * vb * np.sqrt(u4 * u4 + vb * vb)
    rv[sv_j, sv_i] = pgv + corv + (svstr[sv_j, sv_i] - bvstr) * area_v
    return ru, rv


def _step_uv(g, ustp, vstp, Dstp, Dnew, rhs_u, rhs_v, cff1):
    """ubar_new = (ubar(kstp) (Dstp_i + Dstp_i-1) + cff cff1 rhs) / (Dnew_i + Dnew_i-1) on the
    interior faces; walls and the ring stay 0."""
    J, I = Dstp.shape
    un = np.zeros_like(Dstp)
    vn = np.zeros_like(Dstp)
    pm, pn = g["pm"], g["pn"]
    sj, si, sim = slice(1, J - 1), slice(2, I - 1), slice(1, I - 2)
    cff = (pm[sj, si] + pm[sj, sim]) * (pn[sj, si] + pn[sj, sim])
    un[sj, si] = (ustp[sj, si] * (Dstp[sj, si] + Dstp[sj, sim]) + cff * cff1 * rhs_u[sj, si]) / (Dnew[sj, si] + Dnew[sj, sim])
    vj, vi, vjm = slice(2, J - 1), slice(1, I - 1), slice(1, J - 2)
    cffv = (pm[vj, vi] + pm[vjm, vi]) * (pn[vj, vi] + pn[vjm, vi])
    vn[vj, vi] = (vstp[vj, vi] * (Dstp[vj, vi] + Dstp[vjm, vi]) + cffv * cff1 * rhs_v[vj, vi]) / (Dnew[vj, vi] + Dnew[vjm, vi])
    return un, vn


def predictor(g, S, first, dtfast, sustr, svstr, rdrag2, acc=None, step=True):
    """acc: None (no fast-time averages: the 2D-only driver), "reset" (first substep of a
    loop) or (c1, c2), the weights of this substep's accumulation; step False: accumulate
    only (the loop's auxiliary last substep)."""
    zn, un, vn = S.zeta[1], S.ubar[1], S.vbar[1]
    D, DU, DV = _fluxes(g, zn, un, vn)
    if acc is not None:
        if acc[0] == "reset":
            S.Zt_avg1[...] = 0.0
            S.DU_avg1[...] = 0.0
            S.DV_avg1[...] = 0.0
            S.DU_avg2[...] = acc[1] * DU
            S.DV_avg2[...] = acc[1] * DV
        else:
            c1, c2 = acc
            S.Zt_avg1 += c1 * zn
            S.DU_avg1 += c1 * DU
            S.DV_avg1 += c1 * DV
            S.DU_avg2 += c2 * DU
            S.DV_avg2 += c2 * DV
    if not step:
        return
    rz = _rhs_zeta(DU, DV)
    kstp = 1 if first else 0
    cff1 = dtfast if first else 2.0 * dtfast
    zs = S.zeta[kstp]
    znew = zs + g["pm"] * g["pn"] * cff1 * rz
    _ring(znew)
    zwrk = 0.5 * (zs + znew) if first else 0.68 * zn + 0.16 * (zs + znew)
    S.rzeta[1][...] = rz
    ru, rv = _rhs_uv(g, zwrk, D, un, vn, sustr, svstr, rdrag2)
    S.rubar[1][...] = ru
    S.rvbar[1][...] = rv
    Dstp = zs + g["h"]
    Dnew = znew + g["h"]
    up, vp = _step_uv(g, S.ubar[kstp], S.vbar[kstp], Dstp, Dnew, ru, rv,
                      0.5 * dtfast if first else dtfast)
    S.zeta_p[...] = znew
    S.ubar_p[...] = up
    S.vbar_p[...] = vp


def corrector(g, S, first, dtfast, sustr, svstr, rdrag2, c2=None):
    """c2: the weight of this substep's DU_avg2 term (None: no averages)."""
    D, DU, DV = _fluxes(g, S.zeta_p, S.ubar_p, S.vbar_p)
    if c2 is not None:
        S.DU_avg2 += c2 * DU
        S.DV_avg2 += c2 * DV
    rz = _rhs_zeta(DU, DV)
    pmn = g["pm"] * g["pn"]
    if first:
        znew = S.zeta[1] + pmn * dtfast * rz
        zwrk = 0.5 * (S.zeta[1] + znew)
    else:
        znew = S.zeta[1] + pmn * dtfast * ((5.0 / 12.0) * rz + (8.0 / 12.0) * S.rzeta[1]
                                           - (1.0 / 12.0) * S.rzeta[0])
        zwrk = 0.6 * znew + 0.4 * S.zeta_p
    _ring(znew)
    ru, rv = _rhs_uv(g, zwrk, D, S.ubar_p, S.vbar_p, sustr, svstr, rdrag2)
    if first:
        fu, fv, c = ru, rv, 0.5 * dtfast
    else:
        fu = (5.0 / 12.0) * ru + (8.0 / 12.0) * S.rubar[1] - (1.0 / 12.0) * S.rubar[0]
        fv = (5.0 / 12.0) * rv + (8.0 / 12.0) * S.rvbar[1] - (1.0 / 12.0) * S.rvbar[0]
        c = 0.5 * dtfast
    Dstp = S.zeta[1] + g["h"]
    Dnew = znew + g["h"]
    un_, vn_ = _step_uv(g, S.ubar[1], S.vbar[1], Dstp, Dnew, fu, fv, c)
    # n+1 over n-1, then swap: n-1 <- n, n <- n+1
    S.zeta = [S.zeta[1], znew]
    S.ubar = [S.ubar[1], un_]
    S.vbar = [S.vbar[1], vn_]
    S.rzeta = [S.rzeta[1], S.rzeta[0]]
    S.rubar = [S.rubar[1], S.rubar[0]]
    S.rvbar = [S.rvbar[1], S.rvbar[0]]


def loop_weights(iif, W1, W2):
    """(predictor accumulation, corrector DU_avg2 weight) of substep iif (:778-846)."""
    if iif == 1:
        return ("reset", (-1.0 / 12.0) * W2[2]), W2[1]
    return ((W1[iif - 1], (8.0 / 12.0) * W2[iif] - (1.0 / 12.0) * W2[iif + 1]),
            (5.0 / 12.0) * W2[iif])


def barotropic_loop(g, S, nfast, W1, W2, dtfast, sustr, svstr, rdrag2):
    """nfast + 1 substeps: predictor and corrector for iif = 1..nfast, and the accumulating
    predictor of iif = nfast+1 (ROMS does no time stepping in that one)."""
    for iif in range(1, nfast + 2):
        pa, c2 = loop_weights(iif, W1, W2)
        predictor(g, S, iif == 1, dtfast, sustr, svstr, rdrag2, acc=pa, step=iif <= nfast)
        if iif <= nfast:
            corrector(g, S, iif == 1, dtfast, sustr, svstr, rdrag2, c2=c2)


def main2d(g, S, nsteps, dtfast, sustr, svstr, rdrag2, first=True):
    """2D-only driver: predictor + corrector per step, forward/backward Euler on the run's
    first step only, no fast-time averages."""
    for n in range(nsteps):
        f = first and n == 0
        predictor(g, S, f, dtfast, sustr, svstr, rdrag2)
        corrector(g, S, f, dtfast, sustr, svstr, rdrag2)


def volume(g, zeta):
    """Total water volume above the rest level over the interior cells (closed basin)."""
    a = 1.0 / (g["pm"] * g["pn"])
    return float(np.sum((zeta * a)[1:-1, 1:-1]))


# ---------------------------------------------------------------------------------------------
# The baroclinic step with the ROMS-form barotropic loop (the package's semantics "roms"): the
# reference's 3D kernels (restated in oracle/sf_oracle.c, driven as oracle.main3d drives them)
# around this module's barotropic loop, with the surface stress on the top level of the 3D
# right-hand side and closed walls for the 3D velocities.
# ---------------------------------------------------------------------------------------------
class State3D:
    """A ROMS-form 2D State whose arrays sit in zero-guarded parents (the 3D kernels read their
    neighbours past the array ends), beside an oracle.Ocean for the 3D fields."""

    def __init__(self, grid):
        import oracle as orc
        J, I = grid.J, grid.I
        S = State(J, I)
        for name in ("zeta", "ubar", "vbar", "rzeta", "rubar", "rvbar"):
            setattr(S, name, [orc.gzeros((J, I)), orc.gzeros((J, I))])
        for name in ("zeta_p", "ubar_p", "vbar_p", "Zt_avg1", "DU_avg1", "DV_avg1", "DU_avg2",
                     "DV_avg2"):
            setattr(S, name, orc.gzeros((J, I)))
        self.S = S
        self.O = orc.Ocean(grid)
        n3 = (grid.N + 1) * J * I
        self.ru3 = [np.zeros(n3) for _ in range(3)]   # newest first
        self.rv3 = [np.zeros(n3) for _ in range(3)]


def rhs3d(grid, u, v, Huon, Hvom, ru, rv):
    """The ROMS-form 3D momentum right-hand side (m^4/s^2, Hz-weighted as ROMS's ru) at the
    interior faces, 0 elsewhere: Coriolis as ROMS's (UFx = Hz fomn (v_j + v_j+1)/2 at rho
    points, ru += (UFx_i + UFx_i-1)/2; rv -= (VFe_j + VFe_j-1)/2), then second-order centred
    advection of momentum, horizontal (the UV_C2ADVECTION fluxes of the reference's ROMS
    transcription, obsolete/step2d_LF_AM3.h.py:1244-1300, per level with Huon/Hvom for
    DUon/DVom).  The fluxes through the closed walls vanish with the normal transport there.
    The vertical advection is implicit, in the column solve (_column_solve).  The reference's
    runnable rhs3d (rhs_kernels.cpp:71-196) is not this advection (its flux form drops the
    transport factor), so the ROMS-form step has its own."""
    J, I, N = grid.J, grid.I, grid.N
    u3, v3 = u.reshape(N + 1, J, I), v.reshape(N + 1, J, I)
    Hu, Hv = Huon.reshape(N + 1, J, I), Hvom.reshape(N + 1, J, I)
    H3 = grid.Hz.reshape(N, J, I)
    fomn = grid.fomn.reshape(J, I)
    r3u, r3v = ru.reshape(N + 1, J, I), rv.reshape(N + 1, J, I)
    ru[:] = 0.0
    rv[:] = 0.0
    uj, ui = slice(1, J - 1), slice(2, I - 1)          # U faces
    vj, vi = slice(2, J - 1), slice(1, I - 1)          # V faces
    for k in range(N):
        uk, vk, hu, hv = u3[k], v3[k], Hu[k], Hv[k]
        cff = H3[k] * fomn
        UF = np.zeros((J, I))
        UF[:J - 1] = cff[:J - 1] * ((vk[:J - 1] + vk[1:]) * 0.5)
        VF = np.zeros((J, I))
        VF[:, :I - 1] = cff[:, :I - 1] * ((uk[:, :I - 1] + uk[:, 1:]) * 0.5)
        UFx = np.zeros((J, I))                         # at rho (j, i): U faces i and i+1
        UFx[:, :I - 1] = (0.25 * (hu[:, :I - 1] + hu[:, 1:])) * (uk[:, :I - 1] + uk[:, 1:])
        UFe = np.zeros((J, I))                         # at psi (j, i): rows j-1 and j
        UFe[1:, 1:] = (0.25 * (hv[1:, 1:] + hv[1:, :I - 1])) * (uk[1:, 1:] + uk[:J - 1, 1:])
        cor = (UF[uj, ui] + UF[uj, 1:I - 2]) * 0.5
        adv = (UFx[uj, ui] - UFx[uj, 1:I - 2]) + (UFe[2:J, ui] - UFe[uj, ui])
        r3u[k][uj, ui] = cor - adv
        VFx = np.zeros((J, I))                         # at psi (j, i): columns i-1 and i
        VFx[1:, 1:] = (0.25 * (hu[1:, 1:] + hu[:J - 1, 1:])) * (vk[1:, 1:] + vk[1:, :I - 1])
        VFe = np.zeros((J, I))                         # at rho (j, i): V faces j and j+1
        VFe[:J - 1] = (0.25 * (hv[:J - 1] + hv[1:])) * (vk[:J - 1] + vk[1:])
        cor = -((VF[vj, vi] + VF[1:J - 2, vi]) * 0.5)
        adv = (VFx[vj, 2:I] - VFx[vj, vi]) + (VFe[vj, vi] - VFe[1:J - 2, vi])
        r3v[k][vj, vi] = cor - adv


AB3 = ((1.0, 0.0, 0.0), (1.5, -0.5, 0.0), (23.0 / 12.0, -16.0 / 12.0, 5.0 / 12.0))


def ab3_coefficients(k):
    """Adams-Bashforth weights of the right-hand sides at steps n, n-1, n-2 for the k-th step
    since the start (forward Euler, then AB2, then AB3: ROMS's 3D momentum time stepping)."""
    return AB3[min(k, 2)]


def stress3d(grid, u, v, ru, rv, sustr, svstr, rdrag2):
    """Surface and bottom stress on the 3D momentum right-hand side (ROMS's ru includes
    + sustr om_u on_u at k = N and - bustr om_u on_u at k = 1): ru[N-1] += sustr * area and
    ru[0] -= rdrag2 ub sqrt(ub^2 + v_u^2) * area at the interior U faces, with ub the bottom
    level's u and v_u the four-point average of its v (area = 4 / ((pm_i + pm_i-1)(pn_i +
    pn_i-1))); rv likewise at the interior V faces."""
    J, I, N = grid.J, grid.I, grid.N
    pm, pn = grid.pm.reshape(J, I), grid.pn.reshape(J, I)
    r3u, r3v = ru.reshape(N + 1, J, I), rv.reshape(N + 1, J, I)
    u0, v0 = u.reshape(N + 1, J, I)[0], v.reshape(N + 1, J, I)[0]
    sj, si, sim = slice(1, J - 1), slice(2, I - 1), slice(1, I - 2)
    area = 4.0 / ((pm[sj, si] + pm[sj, sim]) * (pn[sj, si] + pn[sj, sim]))
    v4 = 0.25 * (((v0[sj, si] + v0[2:J, si]) + v0[sj, sim]) + v0[2:J, sim])
    ub = u0[sj, si]
    bustr = rdrag2 * ub * np.sqrt(ub * ub + v4 * v4)
    r3u[N - 1][sj, si] = r3u[N - 1][sj, si] + sustr[sj, si] * area
    r3u[0][sj, si] = r3u[0][sj, si] - bustr * area
    vj, vi, vjm = slice(2, J - 1), slice(1, I - 1), slice(1, J - 2)
    area = 4.0 / ((pm[vj, vi] + pm[vjm, vi]) * (pn[vj, vi] + pn[vjm, vi]))
    u4 = 0.25 * (((u0[vj, vi] + u0[vj, 2:I]) + u0[vjm, vi]) + u0[vjm, 2:I])
    vb = v0[vj, vi]
    bvstr = rdrag2 * vb * np.sqrt(u4 * u4 + vb * vb)
    r3v[N - 1][vj, vi] = r3v[N - 1][vj, vi] + svstr[vj, vi] * area
    r3v[0][vj, vi] = r3v[0][vj, vi] - bvstr * area


def _column_solve(grid, u3, rs, c, Hz, Akv, z_r, W, avg, on, sj, si, nj, ni, dt, lamdt):
    """The implicit vertical step of the 3D velocity at the faces (sj, si), whose other rho
    point is (nj, ni): with F_w the upwind vertical advective flux through w level w (w_w x_w-1
    where w_w > 0, w_w x_w where w_w < 0; w_w = fac (W_w + W_w,nbr) / 2, 0 at the bottom and the
    surface) and fac = dt pmU pnU,
      Hzu_k x_k - [viscosity] + (F_k+1 - F_k) = Hzu_k u_k + fac r_k,
    r_k = (c0 ru_k(n) + c1 ru_k(n-1)) + c2 ru_k(n-2) (rs = the three right-hand sides, c their
    Adams-Bashforth weights); the viscosity couples levels k and k+1 through FC_k = -lamdt
    AKU_k+1 / DZ_k (w level k+1; no flux through the surface or the bottom, whose stresses sit
    in ru).  So, with w+ = max(w, 0) and w- = min(w, 0), the lower, main and upper diagonals are
      l_k = FC_k-1 - w+_k,  b_k = (Hzu_k - FC_k - FC_k-1) + (w+_k+1 - w-_k),  u_k = FC_k + w-_k+1,
    an M-matrix at any vertical Courant number, solved by Thomas elimination (backward-Euler
    upwind vertical advection: basin4's thin shelf and slope layers take vertical Courant
    numbers above 1, where the explicit and the implicit centred forms broke down).  Then the
    depth mean is set to the barotropic transport: x_k -= (sum Hzu_k x_k - avg / on) / sum
    Hzu_k (the advective fluxes telescope out of the column sum).  Returns avg / on / sum
    Hzu_k, the barotropic velocity the next loop starts from (step3d_uv.F's coupling)."""
    J, I, N = grid.J, grid.I, grid.N
    pm, pn = grid.pm.reshape(J, I), grid.pn.reshape(J, I)
    H3 = Hz.reshape(N, J, I)
    A3 = Akv.reshape(N + 1, J, I)
    Z3 = z_r.reshape(N, J, I)
    W3 = W.reshape(N + 1, J, I)
    a = (sj, si)
    b = (nj, ni)
    pmU = 0.5 * (pm[a] + pm[b])
    pnU = 0.5 * (pn[a] + pn[b])
    fac = dt * (pmU * pnU)
    hzu = [0.5 * (H3[k][a] + H3[k][b]) for k in range(N)]
    zero = np.zeros_like(pmU)
    FC, WP, WM = [], [zero], [zero]         # w+ and w- on w levels 0..N
    for k in range(N - 1):
        ak = 0.5 * (A3[k + 1][a] + A3[k + 1][b])
        dz = 0.5 * ((Z3[k + 1][a] - Z3[k][a]) + (Z3[k + 1][b] - Z3[k][b]))
        FC.append((-lamdt * ak) / dz)
        wk = fac * (0.5 * (W3[k + 1][a] + W3[k + 1][b]))
        WP.append(np.where(wk > 0.0, wk, 0.0))
        WM.append(np.where(wk < 0.0, wk, 0.0))
    FC.append(zero)
    WP.append(zero)
    WM.append(zero)
    LO, BC, UP, RHS = [], [], [], []
    for k in range(N):
        fcm = FC[k - 1] if k > 0 else zero
        LO.append(fcm - WP[k])
        BC.append(((hzu[k] - FC[k]) - fcm) + (WP[k + 1] - WM[k]))
        UP.append(FC[k] + WM[k + 1])
        r = (c[0] * rs[0][k][a] + c[1] * rs[1][k][a]) + c[2] * rs[2][k][a]
        RHS.append(hzu[k] * u3[k][a] + fac * r)
    for k in range(1, N):
        w = LO[k] / BC[k - 1]
        BC[k] = BC[k] - w * UP[k - 1]
        RHS[k] = RHS[k] - w * RHS[k - 1]
    x = [None] * N
    x[N - 1] = RHS[N - 1] / BC[N - 1]
    for k in range(N - 2, -1, -1):
        x[k] = (RHS[k] - UP[k] * x[k + 1]) / BC[k]
    H = zero.copy()
    Hu = zero.copy()
    for k in range(N):
        H = H + hzu[k]
        Hu = Hu + hzu[k] * x[k]
    target = avg[a] / on[a]
    udiff = (Hu - target) / H
    for k in range(N):
        u3[k][a] = x[k] - udiff
    return target / H


def roms_step3d(grid, S, u, v, ru3, rv3, c, Hz, Akv, z_r, W, dt, lam):
    """The ROMS-form step3d_uv at the interior faces (U: j = 1..J-2, i = 2..I-2; V: j = 2..J-2,
    i = 1..I-2) with the right-hand sides ru3 = (ru(n), ru(n-1), ru(n-2)) weighted by c
    (ab3_coefficients) and lamdt = lam dt, and the barotropic restart: ubar, vbar (slots n and
    scratch) = the new depth-mean velocities at those faces, 0 elsewhere.  W: the vertical
    volume fluxes of the step (omega at its start)."""
    J, I, N = grid.J, grid.I, grid.N
    u3, v3 = u.reshape(N + 1, J, I), v.reshape(N + 1, J, I)
    rs_u = [r.reshape(N + 1, J, I) for r in ru3]
    rs_v = [r.reshape(N + 1, J, I) for r in rv3]
    on_u, om_v = grid.on_u.reshape(J, I), grid.om_v.reshape(J, I)
    lamdt = lam * dt
    ub = np.zeros((J, I))
    vb = np.zeros((J, I))
    sj, si = slice(1, J - 1), slice(2, I - 1)
    ub[sj, si] = _column_solve(grid, u3, rs_u, c, Hz, Akv, z_r, W, S.DU_avg1, on_u, sj, si, sj,
                               slice(1, I - 2), dt, lamdt)
    sj, si = slice(2, J - 1), slice(1, I - 1)
    vb[sj, si] = _column_solve(grid, v3, rs_v, c, Hz, Akv, z_r, W, S.DV_avg1, om_v, sj, si,
                               slice(1, J - 2), si, dt, lamdt)
    for a in (S.ubar[1], S.ubar_p):
        a[...] = ub
    for a in (S.vbar[1], S.vbar_p):
        a[...] = vb


def closed_walls(grid, u, v):
    J, I, N = grid.J, grid.I, grid.N
    u3 = u.reshape(N + 1, J, I)
    v3 = v.reshape(N + 1, J, I)
    u3[:, :, 1] = 0.0
    u3[:, :, I - 1] = 0.0
    v3[:, 1, :] = 0.0
    v3[:, J - 1, :] = 0.0


def main3d(grid, B, st, nsteps, dt, ndtfast, nfast, W1, W2, sustr, svstr, rdrag2, lam=1.0,
           iic0=0, on_step=None):
    """Baroclinic steps in the package's "roms" order: set_maxflux, omega, set_zeta (zeta(n) =
    Zt_avg1), the ROMS-form rhs3d + surface and bottom stress into the newest of three
    right-hand-side slots, the ROMS-form barotropic loop, set_depth, the ROMS-form step3d_uv
    (Adams-Bashforth over the three slots) with the barotropic restart, the reference's
    lateral BCs, closed walls, omega.  AKv stays as it is (no mixing).  st.ru3/st.rv3 hold the
    slots, newest first; the k-th step since the start takes ab3_coefficients(k - iic0)."""
    import oracle as orc
    L = orc.lib()
    S, O = st.S, st.O
    N, J, I = grid.N, grid.J, grid.I
    G = dict(h=grid.h, pm=grid.pm, pn=grid.pn, on_u=grid.on_u, om_v=grid.om_v, fomn=grid.fomn)
    BC = B["zetaBC_bcIdxFieldIdx2"]
    P = orc.P
    dtfast = dt / ndtfast
    O.Zt_avg1[:] = S.Zt_avg1.reshape(-1)
    orc.set_depth(grid, O)
    time = iic0 * dt
    for k in range(nsteps):
        iic = iic0 + k
        L.orc_set_maxflux(grid.ref, P(O.t3("u")), P(O.t3("v")), P(O.Huon), P(O.Hvom), P(grid.Hz))
        L.orc_omega(grid.ref, P(O.W), P(O.Huon), P(O.Hvom), P(grid.z_w), P(BC))
        zt = S.Zt_avg1.reshape(J, I)
        S.zeta[1][...] = zt
        S.zeta_p[...] = zt
        st.ru3.insert(0, st.ru3.pop())
        st.rv3.insert(0, st.rv3.pop())
        ru, rv = st.ru3[0], st.rv3[0]
        rhs3d(grid, O.t3("u"), O.t3("v"), O.Huon, O.Hvom, ru, rv)
        stress3d(grid, O.t3("u"), O.t3("v"), ru, rv, sustr, svstr, rdrag2)
        barotropic_loop(G, S, nfast, W1, W2, dtfast, sustr, svstr, rdrag2)
        O.Zt_avg1[:] = S.Zt_avg1.reshape(-1)
        orc.set_depth(grid, O)
        roms_step3d(grid, S, O.t3("u"), O.t3("v"), st.ru3, st.rv3, ab3_coefficients(k), grid.Hz,
                    O.AKv, grid.z_r, O.W, dt, lam)
        L.orc_lateral_uv_bc(grid.ref, orc.D(time), P(O.t3("u")), P(O.t3("v")),
                            P(B["vvelBC_bcIdxFieldIdx2"]), P(B["uvelBC_bcIdxFieldType"]),
                            P(B["vvelBC_bcIdxFieldType"]))
        closed_walls(grid, O.t3("u"), O.t3("v"))
        L.orc_omega(grid.ref, P(O.W), P(O.Huon), P(O.Hvom), P(grid.z_w), P(BC))
        time += dt
        if on_step is not None:
            on_step(iic + 1, S, O)
