"""A small stratified, sheared, wind-driven basin for the GLS closure tests."""
import numpy as np

from sailfish_b200 import host


def make(Lm=14, Mm=10, N=20, seed=7, wind=1.0e-4):
    rng = np.random.default_rng(seed)
    L, M = Lm + 1, Mm + 1
    I, J = L + 1, M + 1
    s2 = I * J
    jj, ii = np.meshgrid(np.arange(J), np.arange(I), indexing="ij")
    h = (60.0 + 40.0 * np.tanh((jj - J / 2) / 3.0) + 2.0 * ii).reshape(-1)
    sc_r, sc_w, Cs_r, Cs_w = host.set_coords(N, 4, 5.0, 0.4)
    hc = 20.0
    zeta = 0.05 * rng.standard_normal(s2)
    z_w = np.zeros((N + 1, s2))
    z_r = np.zeros((N, s2))
    for k in range(N + 1):
        z_w[k] = zeta + (zeta + h) * (hc * sc_w[k] + Cs_w[k] * h) / (hc + h)
    for k in range(N):
        z_r[k] = zeta + (zeta + h) * (hc * sc_r[k] + Cs_r[k] * h) / (hc + h)
    Hz = z_w[1:] - z_w[:-1]
    u = np.zeros((N + 1, s2))
    v = np.zeros((N + 1, s2))
    u[:N] = 0.3 * (1.0 + z_r / h) + 0.02 * rng.standard_normal((N, s2))
    v[:N] = -0.1 * (1.0 + z_r / h) + 0.02 * rng.standard_normal((N, s2))
    # linear EOS with T = 4 + 20 exp(z/500): N^2 = g alpha dT/dz (alpha = 1.7e-4)
    bvf = 10.0 * 1.7e-4 * (20.0 / 500.0) * np.exp(z_w / 500.0)
    bvf[:, ::7] *= -0.3        # a few convectively unstable points
    tke = 1.0e-4 * (1.0 + rng.random((N + 1, s2)))
    Lsc = 0.5 + rng.random((N + 1, s2))
    gls = 0.5477 ** 3 * tke ** 1.5 / Lsc
    Akv = 1.0e-3 * (1.0 + rng.random((N + 1, s2)))
    Akt = 1.0e-4 * (1.0 + rng.random((N + 1, s2)))
    Akk = 1.0e-3 * (1.0 + rng.random((N + 1, s2)))
    Akp = 1.0e-3 * (1.0 + rng.random((N + 1, s2)))
    sustr = np.full(s2, wind)
    svstr = np.full(s2, 0.2 * wind)
    return dict(I=I, J=J, N=N, h=h, sc_r=sc_r, sc_w=sc_w, Cs_r=Cs_r, Cs_w=Cs_w, hc=hc, z_w=z_w,
                z_r=z_r, Hz=Hz, u=u, v=v, bvf=bvf, tke=tke, gls=gls, Akv=Akv, Akt=Akt, Akk=Akk,
                Akp=Akp, Lscale=Lsc, sustr=sustr, svstr=svstr)
