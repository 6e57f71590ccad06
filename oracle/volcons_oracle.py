"""obc_volcons restated in Python (TEST INFRASTRUCTURE: the oracle).

nonlinear/obc_volcons.py:6-69 is ROMS pseudo-code in the reference (not runnable): the
cross-section area and volume flux through the open boundary edges, ubar_xs = flux / area,
and conserve_mass_tile's correction of the normal barotropic velocity on those edges.  Sums
here are exact (math.fsum), the standard the compensated device sums are held to.  Parity
unpinned by reference outputs.

Edges: W=1, E=2, S=4, N=8.  Fields are flat (M+1)*(L+1) in the reference's layout (i fastest).
"""
import math

import numpy as np


def edge_terms(I, J, zeta, h, ubar, vbar, on_u, om_v, edges):
    """(cff, signed cff*velocity) of every open-edge face, in the order W, E, S, N."""
    L, M = I - 1, J - 1
    D = (np.asarray(zeta, np.float64) + np.asarray(h, np.float64)).reshape(J, I)
    u2, v2 = np.asarray(ubar, np.float64).reshape(J, I), np.asarray(vbar, np.float64).reshape(J, I)
    ou, ov = np.asarray(on_u, np.float64).reshape(J, I), np.asarray(om_v, np.float64).reshape(J, I)
    area, flux = [], []
    js, is_ = range(1, M), range(1, L)
    if edges & 1:
        for j in js:
            c = 0.5 * (D[j, 0] + D[j, 1]) * ou[j, 1]
            area.append(c)
            flux.append(c * u2[j, 1])
    if edges & 2:
        for j in js:
            c = 0.5 * (D[j, L - 1] + D[j, L]) * ou[j, L]
            area.append(c)
            flux.append(-c * u2[j, L])
    if edges & 4:
        for i in is_:
            c = 0.5 * (D[0, i] + D[1, i]) * ov[1, i]
            area.append(c)
            flux.append(c * v2[1, i])
    if edges & 8:
        for i in is_:
            c = 0.5 * (D[M - 1, i] + D[M, i]) * ov[M, i]
            area.append(c)
            flux.append(-c * v2[M, i])
    return area, flux


def obc_volcons(I, J, zeta, h, ubar, vbar, on_u, om_v, edges):
    """(area, flux, ubar_xs) with exact sums."""
    area, flux = edge_terms(I, J, zeta, h, ubar, vbar, on_u, om_v, edges)
    a, f = math.fsum(area), math.fsum(flux)
    return a, f, (f / a if a > 0 else 0.0)


def conserve_mass(I, J, ubar, vbar, xs, edges):
    """conserve_mass_tile: ubar -= xs on W, += xs on E; vbar -= xs on S, += xs on N."""
    L, M = I - 1, J - 1
    u2 = np.array(ubar, np.float64).reshape(J, I)
    v2 = np.array(vbar, np.float64).reshape(J, I)
    if edges & 1:
        u2[1:M, 1] -= xs
    if edges & 2:
        u2[1:M, L] += xs
    if edges & 4:
        v2[1, 1:L] -= xs
    if edges & 8:
        v2[M, 1:L] += xs
    return u2.ravel(), v2.ravel()
