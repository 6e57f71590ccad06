// ROMS-form barotropic step (the "roms" semantics): the free-surface / depth-integrated
// momentum step of ROMS's step2d_LF_AM3, which the reference carries only as untranslated
// Fortran (obsolete/step2d_LF_AM3.h.py), with its 2D Coriolis (:1503-1530), surface stress
// (:2598-2612), quadratic bottom drag (nonlinear/set_vbc.py:16-41) and the fast-time averages
// Zt_avg1, DU_avg1/2, DV_avg1/2 (:778-846), for closed rectangular basins.  It exists beside
// the reference-semantics kernels because the benchmark configurations need forcing, Coriolis
// and a stable step, none of which the reference's runnable 2D kernels have.
//
// Divisions go through ddiv: IEEE in FP64, the fast FP32 division (__fdividef) in FP32.
//
// Index conventions as the rest of the package: flat p = j*I + i over (M+1) x (L+1) rho points;
// ubar(p) on the west face of rho p, vbar(p) on its south face; interior rho i = 1..I-2,
// j = 1..J-2; interior U faces i = 2..I-2 (walls i = 1, I-1), V faces j = 2..J-2.
//
// A substep is four launches: the predictor's free surface (k_roms_zeta, phase 0), its
// momentum (k_roms_mom, phase 0), the corrector's free surface (phase 1) and momentum
// (phase 1).  Time levels: slots b (n-1), n and p (the predicted n+1*); the corrector writes
// n+1 into b and the host swaps b and n.  Every expression keeps the operand order of the
// oracle's restatement (oracle/roms_oracle.py), so the FP64 build (no FMA contraction)
// reproduces it bit for bit; the fast-time averages are FP64 in both precisions.
#pragma once

namespace sf {


// DUon at the U face p (0 on column 0) and DVom at the V face p (0 on row 0), from zeta, ubar, vbar
template <typename R>
__device__ __forceinline__ R roms_du(const Geo<R> &g, const R *z, const R *u, long p, int i) {
    if (i < 1) return R(0);
    const R Dp = z[p] + g.h[p], Dw = z[p - 1] + g.h[p - 1];
    return (u[p] * (R(0.5) * (Dp + Dw))) * g.on_u[p];
}
template <typename R>
__device__ __forceinline__ R roms_dv(const Geo<R> &g, const R *z, const R *v, long p, int j) {
    if (j < 1) return R(0);
    const R Dp = z[p] + g.h[p], Ds = z[p - g.I] + g.h[p - g.I];
    return (v[p] * (R(0.5) * (Dp + Ds))) * g.om_v[p];
}
// rhs_zeta at interior rho q: (DUon_q - DUon_q+1) + (DVom_q - DVom_q+I)
template <typename R>
__device__ __forceinline__ R roms_rz(const Geo<R> &g, const R *z, const R *u, const R *v, long q,
                                     int i, int j) {
    return (roms_du(g, z, u, q, i) - roms_du(g, z, u, q + 1, i + 1)) +
           (roms_dv(g, z, v, q, j) - roms_dv(g, z, v, q + g.I, j + 1));
}

// Free surface of a phase at rho p.  Ring nodes take the value of the nearest interior node
// (zero gradient at closed walls), computed here from the inputs.
template <typename R>
__device__ __forceinline__ void roms_zeta_at(const Geo<R> &g, const RomsArgs<R> &a, const long p) {
    if (p >= g.s2) return;
    const int j = fdiv((int)p, g.dI), i = (int)p - j * g.I;
    const long I = g.I;
    if (a.acc) {   // the fast-time averages at rho p, its west U face and its south V face
        const R *z = a.phase == 0 ? a.zn : a.zp;
        const R *u = a.phase == 0 ? a.un : a.up;
        const R *v = a.phase == 0 ? a.vn : a.vp;
        const double du = (double)roms_du(g, z, u, p, i), dv = (double)roms_dv(g, z, v, p, j);
        if (a.phase == 0) {
            if (a.acc == 2) {
                a.Zt[p] = 0.0;
                a.DU1[p] = 0.0;
                a.DV1[p] = 0.0;
                a.DU2[p] = a.c2 * du;
                a.DV2[p] = a.c2 * dv;
            } else {
                a.Zt[p] = a.Zt[p] + a.c1 * (double)z[p];
                a.DU1[p] = a.DU1[p] + a.c1 * du;
                a.DV1[p] = a.DV1[p] + a.c1 * dv;
                a.DU2[p] = a.DU2[p] + a.c2 * du;
                a.DV2[p] = a.DV2[p] + a.c2 * dv;
            }
        } else {
            a.DU2[p] = a.DU2[p] + a.c2 * du;
            a.DV2[p] = a.DV2[p] + a.c2 * dv;
        }
    }
    if (!a.step) return;
    const int qi = i < 1 ? 1 : (i > g.I - 2 ? g.I - 2 : i);
    const int qj = j < 1 ? 1 : (j > g.J - 2 ? g.J - 2 : j);
    const long q = (long)qj * I + qi;
    const R pmn = g.pm[q] * g.pn[q];
    R znew;
    if (a.phase == 0) {
        const R rz = roms_rz(g, a.zn, a.un, a.vn, q, qi, qj);
        const R cff1 = a.first ? (R)a.dtfast : (R)(2.0 * a.dtfast);
        znew = a.zkstp[q] + (pmn * cff1) * rz;
        if (q == p) a.rz_n[p] = rz;
    } else {
        const R rz = roms_rz(g, a.zp, a.up, a.vp, q, qi, qj);
        const R dt = (R)a.dtfast;
        if (a.first)
            znew = a.zn[q] + (pmn * dt) * rz;
        else
            znew = a.zn[q] + (pmn * dt) * ((R(5.0 / 12.0) * rz + R(8.0 / 12.0) * a.rz_n[q]) -
                                          R(1.0 / 12.0) * a.rz_b[q]);
    }
    a.zout[p] = znew;
    if (a.phase == 0 && q != p) a.rz_n[p] = R(0);
}

// The pressure-gradient surface zwrk of a phase at rho q (zout holds the phase's new zeta).
template <typename R>
__device__ __forceinline__ R roms_zwrk(const RomsArgs<R> &a, long q) {
    const R znew = a.zout[q];
    if (a.first) return R(0.5) * (a.zkstp[q] + znew);
    if (a.phase == 0) return R(0.68) * a.zn[q] + R(0.16) * (a.zkstp[q] + znew);
    return R(0.6) * znew + R(0.4) * a.zp[q];
}

// Momentum of a phase at the U and V faces of p (0 on walls and the ring).
template <typename R>
__device__ __forceinline__ void roms_mom_at(const Geo<R> &g, const RomsArgs<R> &a, const long p) {
    if (p >= g.s2) return;
    const int j = fdiv((int)p, g.dI), i = (int)p - j * g.I;
    const long I = g.I;
    const R *h = g.h;
    const R cffg = R(0.5 * 10.0);                    // 0.5 g, g = 10 (mod_constants.py:26)
    const R *zr = a.zrhs, *ur = a.urhs, *vr = a.vrhs;
    const R rdrag2 = (R)a.rdrag2;
    const R cdt = a.first ? (R)(0.5 * a.dtfast) : (a.phase == 0 ? (R)a.dtfast : (R)(0.5 * a.dtfast));
    // U face p
    R unew = R(0), runew = R(0);
    if (i >= 2 && i <= g.I - 2 && j >= 1 && j <= g.J - 2) {
        const R gp = roms_zwrk(a, p), gw = roms_zwrk(a, p - 1);
        const R gp2 = gp * gp, gw2 = gw * gw;
        const R pg = (cffg * g.on_u[p]) * ((h[p - 1] + h[p]) * (gw - gp) + (gw2 - gp2));
        const R UFp = ((R(0.5) * (zr[p] + h[p])) * g.fomn[p]) * (vr[p] + vr[p + I]);
        const R UFw = ((R(0.5) * (zr[p - 1] + h[p - 1])) * g.fomn[p - 1]) * (vr[p - 1] + vr[p - 1 + I]);
        const R cor = R(0.5) * (UFp + UFw);
        const R area = ddiv(R(4.0), (g.pm[p] + g.pm[p - 1]) * (g.pn[p] + g.pn[p - 1]));
        const R v4 = R(0.25) * (((vr[p] + vr[p + I]) + vr[p - 1]) + vr[p - 1 + I]);
        const R ub = ur[p];
        const R bustr = (rdrag2 * ub) * sqrt(ub * ub + v4 * v4);
        const R ru = (pg + cor) + (a.sustr[p] - bustr) * area;
        R f = ru;
        if (a.phase == 0) runew = ru;
        else if (!a.first) f = (R(5.0 / 12.0) * ru + R(8.0 / 12.0) * a.ru_n[p]) - R(1.0 / 12.0) * a.ru_b[p];
        const R cff = (g.pm[p] + g.pm[p - 1]) * (g.pn[p] + g.pn[p - 1]);
        const R Ds = (a.zkstp[p] + h[p]) + (a.zkstp[p - 1] + h[p - 1]);
        const R Dn = (a.zout[p] + h[p]) + (a.zout[p - 1] + h[p - 1]);
        unew = ddiv(a.ukstp[p] * Ds + (cff * cdt) * f, Dn);
    }
    a.uout[p] = unew;
    if (a.phase == 0) a.ru_n[p] = runew;
    // V face p
    R vnew = R(0), rvnew = R(0);
    if (j >= 2 && j <= g.J - 2 && i >= 1 && i <= g.I - 2) {
        const R gp = roms_zwrk(a, p), gs = roms_zwrk(a, p - I);
        const R gp2 = gp * gp, gs2 = gs * gs;
        const R pg = (cffg * g.om_v[p]) * ((h[p - I] + h[p]) * (gs - gp) + (gs2 - gp2));
        const R VFp = ((R(0.5) * (zr[p] + h[p])) * g.fomn[p]) * (ur[p] + ur[p + 1]);
        const R VFs = ((R(0.5) * (zr[p - I] + h[p - I])) * g.fomn[p - I]) * (ur[p - I] + ur[p - I + 1]);
        const R cor = R(-0.5) * (VFp + VFs);
        const R area = ddiv(R(4.0), (g.pm[p] + g.pm[p - I]) * (g.pn[p] + g.pn[p - I]));
        const R u4 = R(0.25) * (((ur[p] + ur[p + 1]) + ur[p - I]) + ur[p - I + 1]);
        const R vb = vr[p];
        const R bvstr = (rdrag2 * vb) * sqrt(u4 * u4 + vb * vb);
        const R rv = (pg + cor) + (a.svstr[p] - bvstr) * area;
        R f = rv;
        if (a.phase == 0) rvnew = rv;
        else if (!a.first) f = (R(5.0 / 12.0) * rv + R(8.0 / 12.0) * a.rv_n[p]) - R(1.0 / 12.0) * a.rv_b[p];
        const R cff = (g.pm[p] + g.pm[p - I]) * (g.pn[p] + g.pn[p - I]);
        const R Ds = (a.zkstp[p] + h[p]) + (a.zkstp[p - I] + h[p - I]);
        const R Dn = (a.zout[p] + h[p]) + (a.zout[p - I] + h[p - I]);
        vnew = ddiv(a.vkstp[p] * Ds + (cff * cdt) * f, Dn);
    }
    a.vout[p] = vnew;
    if (a.phase == 0) a.rv_n[p] = rvnew;
}

// The ROMS-form 3D momentum right-hand side at the interior faces (U: j = 1..J-2, i = 2..I-2;
// V: j = 2..J-2, i = 1..I-2), 0 elsewhere, every level: Coriolis as ROMS's (and the
// reference's addCoriolis), then second-order centred advection of momentum: horizontal
// fluxes UFx = (Huon_i + Huon_i+1)/4 (u_i + u_i+1) at rho points and UFe = (Hvom_i +
// Hvom_i-1)/4 (u_j + u_j-1) at psi points (the UV_C2ADVECTION form of the reference's ROMS
// transcription, obsolete/step2d_LF_AM3.h.py:1244-1300, per level), V alike; the vertical
// advection is implicit, in the column solve (roms_column).  One thread per rho point p (its
// west U face and south V face), levels in order; the expressions keep the oracle's operand
// order (oracle/roms_oracle.py, rhs3d).
template <typename R>
__device__ __forceinline__ void roms_rhs3d_at(const Geo<R> &g, const R *__restrict__ u,
                                              const R *__restrict__ v, const R *__restrict__ Hu,
                                              const R *__restrict__ Hv, const R *__restrict__ Hz,
                                              R *__restrict__ ru, R *__restrict__ rv,
                                              const long p) {
    if (p >= g.s2) return;
    const int j = fdiv((int)p, g.dI), i = (int)p - j * g.I;
    const long I = g.I, s2 = g.s2;
    const int N = g.N;
    const bool uf = i >= 2 && i <= g.I - 2 && j >= 1 && j <= g.J - 2;
    const bool vf = j >= 2 && j <= g.J - 2 && i >= 1 && i <= g.I - 2;
    const R *fomn = g.fomn;
    for (int k = 0; k <= N; ++k) {
        const long o = (long)k * s2;
        R tu = R(0), tv = R(0);
        if (k < N && uf) {
            const R *uk = u + o, *vk = v + o, *hu = Hu + o, *hv = Hv + o, *hz = Hz + o;
            const R UFp = (hz[p] * fomn[p]) * ((vk[p] + vk[p + I]) * R(0.5));
            const R UFw = (hz[p - 1] * fomn[p - 1]) * ((vk[p - 1] + vk[p - 1 + I]) * R(0.5));
            const R cor = (UFp + UFw) * R(0.5);
            const R Xp = (R(0.25) * (hu[p] + hu[p + 1])) * (uk[p] + uk[p + 1]);
            const R Xw = (R(0.25) * (hu[p - 1] + hu[p])) * (uk[p - 1] + uk[p]);
            const R En = (R(0.25) * (hv[p + I] + hv[p + I - 1])) * (uk[p + I] + uk[p]);
            const R Es = (R(0.25) * (hv[p] + hv[p - 1])) * (uk[p] + uk[p - I]);
            tu = cor - ((Xp - Xw) + (En - Es));
        }
        if (k < N && vf) {
            const R *uk = u + o, *vk = v + o, *hu = Hu + o, *hv = Hv + o, *hz = Hz + o;
            const R VFp = (hz[p] * fomn[p]) * ((uk[p] + uk[p + 1]) * R(0.5));
            const R VFs = (hz[p - I] * fomn[p - I]) * ((uk[p - I] + uk[p - I + 1]) * R(0.5));
            const R cor = -((VFp + VFs) * R(0.5));
            const R Xe = (R(0.25) * (hu[p + 1] + hu[p + 1 - I])) * (vk[p + 1] + vk[p]);
            const R Xw = (R(0.25) * (hu[p] + hu[p - I])) * (vk[p] + vk[p - 1]);
            const R Ep = (R(0.25) * (hv[p] + hv[p + I])) * (vk[p] + vk[p + I]);
            const R Es = (R(0.25) * (hv[p - I] + hv[p])) * (vk[p - I] + vk[p]);
            tv = cor - ((Xe - Xw) + (Ep - Es));
        }
        ru[o + p] = tu;
        rv[o + p] = tv;
    }
}

// Surface and bottom stress on the 3D momentum right-hand side (ROMS's ru includes
// + sustr om_u on_u at k = N and - bustr om_u on_u at k = 1): ru[N-1] += sustr * area and
// ru[0] -= rdrag2 ub sqrt(ub^2 + v_u^2) * area at the interior U faces, ub the bottom level's u,
// v_u the four-point average of its v; rv likewise at the interior V faces.
template <typename R>
__device__ __forceinline__ void roms_stress3d_at(const Geo<R> &g, const R *__restrict__ u,
                                                 const R *__restrict__ v, R *__restrict__ ru,
                                                 R *__restrict__ rv, const R *__restrict__ sustr,
                                                 const R *__restrict__ svstr, R rdrag2,
                                                 const long p) {
    if (p >= g.s2) return;
    const int j = fdiv((int)p, g.dI), i = (int)p - j * g.I;
    const long I = g.I, o = (long)(g.N - 1) * g.s2 + p;
    if (i >= 2 && i <= g.I - 2 && j >= 1 && j <= g.J - 2) {
        const R area = ddiv(R(4.0), (g.pm[p] + g.pm[p - 1]) * (g.pn[p] + g.pn[p - 1]));
        const R v4 = R(0.25) * (((v[p] + v[p + I]) + v[p - 1]) + v[p + I - 1]);
        const R ub = u[p];
        const R bustr = rdrag2 * ub * sqrt(ub * ub + v4 * v4);
        ru[o] = ru[o] + sustr[p] * area;
        ru[p] = ru[p] - bustr * area;
    }
    if (j >= 2 && j <= g.J - 2 && i >= 1 && i <= g.I - 2) {
        const R area = ddiv(R(4.0), (g.pm[p] + g.pm[p - I]) * (g.pn[p] + g.pn[p - I]));
        const R u4 = R(0.25) * (((u[p] + u[p + 1]) + u[p - I]) + u[p - I + 1]);
        const R vb = v[p];
        const R bvstr = rdrag2 * vb * sqrt(u4 * u4 + vb * vb);
        rv[o] = rv[o] + svstr[p] * area;
        rv[p] = rv[p] - bvstr * area;
    }
}

// The ROMS-form step3d_uv for one face column (d = 1: U face, d = I: V face): with F_w the
// upwind vertical advective flux through w level w (w_w x_w-1 where w_w > 0, w_w x_w where
// w_w < 0; w_w = fac (W_w + W_w,nbr) / 2, 0 at the bottom and the surface), fac = dt pmU pnU,
//   Hzu_k x_k - [viscosity] + (F_k+1 - F_k) = Hzu_k u_k + fac r_k,
// r_k = (c0 ru_k(n) + c1 ru_k(n-1)) + c2 ru_k(n-2) (Adams-Bashforth), the viscosity through
// FC_k = -lamdt AKU_k+1 / DZ_k on the interface between levels k and k+1 (w level k+1; no flux
// through the surface or the bottom, whose stresses are in ru): the lower, main and upper
// diagonals l_k = FC_k-1 - w+_k, b_k = (Hzu_k - FC_k - FC_k-1) + (w+_k+1 - w-_k),
// u_k = FC_k + w-_k+1 (an M-matrix at any vertical Courant number: backward-Euler upwind
// vertical advection).  Thomas elimination in R, then the depth mean set to the barotropic
// transport with FP64 sums: x_k -= (sum Hzu x - avg/on) / sum Hzu.  Returns the new depth-mean
// velocity avg/on/sum Hzu.
template <typename R>
struct RomsRhs {
    const R *r0, *r1, *r2;   // right-hand sides at n, n-1, n-2
};

template <typename R>
__device__ __forceinline__ double roms_column(const Geo<R> &g, long p, long d, R *__restrict__ u,
                                              RomsRhs<R> rs, R c0, R c1, R c2,
                                              const R *__restrict__ Hz,
                                              const R *__restrict__ Akv, const R *__restrict__ z_r,
                                              const R *__restrict__ W, double avg, R on, R dt,
                                              R lamdt) {
    const long s2 = g.s2;
    const int N = g.N;
    // the eliminated main and upper diagonals and right-hand side per level; the viscous
    // coefficients FC, the vertical fluxes and the layer thicknesses are formed level by level
    // (those of the level below carried in registers) and the thicknesses formed again for the
    // sums: the same operations, in the same order, as storing them
    R bc[kRomsMaxN], up[kRomsMaxN], rhs[kRomsMaxN];
    const R pmU = R(0.5) * (g.pm[p] + g.pm[p - d]);
    const R pnU = R(0.5) * (g.pn[p] + g.pn[p - d]);
    const R fac = dt * (pmU * pnU);
    auto wplus = [](R w) { return w > R(0) ? w : R(0); };
    auto wminus = [](R w) { return w < R(0) ? w : R(0); };
    R fcm = R(0), wk = R(0);   // FC of the level below, the flux through this level's bottom
    // the levels' loads (independent of the elimination) issued kC levels at a time: one
    // exposed load latency per chunk instead of per level (basin4: 4.70 ms with one level at a
    // time, 3.58 with 4, 4.22 with 8 at 128 registers)
    constexpr int kC = 4;
    for (int k0 = 0; k0 < N; k0 += kC) {
        R hz0[kC], hz1[kC], ak0[kC], ak1[kC], zr0[kC], zr1[kC], zq0[kC], zq1[kC], w0[kC], w1[kC],
            q0[kC], q1[kC], q2[kC], uo[kC];
#pragma unroll
        for (int c = 0; c < kC; ++c) {
            const int k = k0 + c < N ? k0 + c : N - 1;
            const int kn = k + 1 < N ? k + 1 : N - 1;   // the next level (unused at the top)
            const long o = (long)k * s2 + p, on_ = (long)kn * s2 + p;
            hz0[c] = Hz[o];
            hz1[c] = Hz[o - d];
            ak0[c] = Akv[on_];
            ak1[c] = Akv[on_ - d];
            zr0[c] = z_r[on_];
            zr1[c] = z_r[o];
            zq0[c] = z_r[on_ - d];
            zq1[c] = z_r[o - d];
            w0[c] = W[on_];
            w1[c] = W[on_ - d];
            q0[c] = rs.r0[o];
            q1[c] = rs.r1[o];
            q2[c] = rs.r2[o];
            uo[c] = u[o];
        }
#pragma unroll
        for (int c = 0; c < kC; ++c) {
            const int k = k0 + c;
            if (k >= N) break;
            const R hzu = R(0.5) * (hz0[c] + hz1[c]);
            R fck, wk1;
            if (k < N - 1) {
                const R ak = R(0.5) * (ak0[c] + ak1[c]);
                const R dz = R(0.5) * ((zr0[c] - zr1[c]) + (zq0[c] - zq1[c]));
                fck = ddiv(-lamdt * ak, dz);
                wk1 = fac * (R(0.5) * (w0[c] + w1[c]));
            } else {
                fck = R(0);
                wk1 = R(0);
            }
            const R fcm_k = k > 0 ? fcm : R(0);
            R b = ((hzu - fck) - fcm_k) + (wplus(wk1) - wminus(wk));
            up[k] = fck + wminus(wk1);
            const R r = (c0 * q0[c] + c1 * q1[c]) + c2 * q2[c];
            R x = hzu * uo[c] + fac * r;
            if (k > 0) {
                const R w = ddiv(fcm_k - wplus(wk), bc[k - 1]);
                b = b - w * up[k - 1];
                x = x - w * rhs[k - 1];
            }
            bc[k] = b;
            rhs[k] = x;
            fcm = fck;
            wk = wk1;
        }
    }
    rhs[N - 1] = ddiv(rhs[N - 1], bc[N - 1]);          // x overwrites rhs
    for (int k = N - 2; k >= 0; --k) rhs[k] = ddiv(rhs[k] - up[k] * rhs[k + 1], bc[k]);
    double H = 0.0, Hu = 0.0;
    constexpr int kS = 8;   // the thicknesses' loads kS levels at a time
    for (int k0 = 0; k0 < N; k0 += kS) {
        R ha[kS], hb[kS];
#pragma unroll
        for (int c = 0; c < kS; ++c) {
            const long o = (long)(k0 + c < N ? k0 + c : N - 1) * s2 + p;
            ha[c] = Hz[o];
            hb[c] = Hz[o - d];
        }
#pragma unroll
        for (int c = 0; c < kS; ++c) {
            if (k0 + c >= N) break;
            const R hzu = R(0.5) * (ha[c] + hb[c]);
            H = H + (double)hzu;
            Hu = Hu + (double)hzu * (double)rhs[k0 + c];
        }
    }
    const double target = avg / (double)on;
    const double udiff = (Hu - target) / H;
    for (int k = 0; k < N; ++k) u[(long)k * s2 + p] = (R)((double)rhs[k] - udiff);
    return target / H;
}

// The ROMS-form step3d_uv over the interior faces (U: j = 1..J-2, i = 2..I-2; V: j = 2..J-2,
// i = 1..I-2), one thread per face column (a rho point's west U column or its south V
// column; ensembles: both, one after the other), and the barotropic restart: ubar, vbar in
// slots n and scratch = the new depth-mean velocities at those faces, 0 elsewhere.
// t < s2: the U column (west face) of rho point t; s2 <= t < 2 s2: the V column (south face)
// of rho point t - s2.
template <typename R>
__device__ __forceinline__ void roms_step3d_at(const Geo<R> &g, R *__restrict__ u,
                                               R *__restrict__ v, RomsRhs<R> ru, RomsRhs<R> rv,
                                               R c0, R c1, R c2, R *__restrict__ ubar_n,
                                               R *__restrict__ vbar_n, R *__restrict__ ubar_s,
                                               R *__restrict__ vbar_s, const R *__restrict__ Hz,
                                               const R *__restrict__ Akv,
                                               const R *__restrict__ z_r,
                                               const R *__restrict__ W,
                                               const double *__restrict__ DU,
                                               const double *__restrict__ DV, R dt, R lamdt,
                                               const long t) {
    if (t >= 2 * g.s2) return;
    const bool vcol = t >= g.s2;
    const long p = vcol ? t - g.s2 : t;
    const int j = fdiv((int)p, g.dI), i = (int)p - j * g.I;
    R bar = R(0);
    if (!vcol) {
        if (i >= 2 && i <= g.I - 2 && j >= 1 && j <= g.J - 2)
            bar = (R)roms_column(g, p, 1, u, ru, c0, c1, c2, Hz, Akv, z_r, W, DU[p], g.on_u[p], dt,
                                 lamdt);
        ubar_n[p] = bar;
        ubar_s[p] = bar;
    } else {
        if (j >= 2 && j <= g.J - 2 && i >= 1 && i <= g.I - 2)
            bar = (R)roms_column(g, p, g.I, v, rv, c0, c1, c2, Hz, Akv, z_r, W, DV[p], g.om_v[p],
                                 dt, lamdt);
        vbar_n[p] = bar;
        vbar_s[p] = bar;
    }
}

// Closed walls for the 3D velocities: u = 0 on the U wall faces (i = 1, I-1), v = 0 on the V
// wall faces (j = 1, J-1), every level.
template <typename R>
__device__ __forceinline__ void roms_walls3d_at(const Geo<R> &g, R *__restrict__ u,
                                                R *__restrict__ v, const long p) {
    if (p >= g.s2) return;
    const int j = fdiv((int)p, g.dI), i = (int)p - j * g.I;
    const bool uw = (i == 1 || i == g.I - 1), vw = (j == 1 || j == g.J - 1);
    if (!uw && !vw) return;
    for (int k = 0; k <= g.N; ++k) {
        if (uw) u[(long)k * g.s2 + p] = R(0);
        if (vw) v[(long)k * g.s2 + p] = R(0);
    }
}

// Kernels: a single grid (one thread per flat point) and ensembles (a block map gives each
// block its member and its block within the member; the member's fields are offset in the
// pools: 2D fields by off2, fields of N+1 levels by off3, of N levels by offN).
template <typename R>
struct MemberAt {
    Geo<R> g;
    long o2, o3, oN, p;
};
template <typename R>
__device__ __forceinline__ MemberAt<R> member_at(const Member<R> *mt, const int2 *bm, int bs) {
    const int2 mb = bm[blockIdx.x];
    const Member<R> &M = mt[mb.x];
    return MemberAt<R>{M.g, M.off2, M.off3, M.offN, (long)mb.y * bs + threadIdx.x};
}
template <typename T>
__device__ __forceinline__ T *at(T *x, long o) { return x ? x + o : x; }
template <typename R>
__device__ __forceinline__ RomsArgs<R> roms_args_at(const RomsArgs<R> &a, long o) {
    RomsArgs<R> b = a;
    b.zb = at(a.zb, o); b.zn = at(a.zn, o); b.zp = at(a.zp, o);
    b.ub = at(a.ub, o); b.un = at(a.un, o); b.up = at(a.up, o);
    b.vb = at(a.vb, o); b.vn = at(a.vn, o); b.vp = at(a.vp, o);
    b.zout = at(a.zout, o); b.uout = at(a.uout, o); b.vout = at(a.vout, o);
    b.zkstp = at(a.zkstp, o); b.ukstp = at(a.ukstp, o); b.vkstp = at(a.vkstp, o);
    b.zrhs = at(a.zrhs, o); b.urhs = at(a.urhs, o); b.vrhs = at(a.vrhs, o);
    b.rz_n = at(a.rz_n, o); b.ru_n = at(a.ru_n, o); b.rv_n = at(a.rv_n, o);
    b.rz_b = at(a.rz_b, o); b.ru_b = at(a.ru_b, o); b.rv_b = at(a.rv_b, o);
    b.sustr = at(a.sustr, o); b.svstr = at(a.svstr, o);
    b.Zt = at(a.Zt, o); b.DU1 = at(a.DU1, o); b.DV1 = at(a.DV1, o);
    b.DU2 = at(a.DU2, o); b.DV2 = at(a.DV2, o);
    return b;
}

// The barotropic phases are launched with programmatic dependent launch (as the reference
// form's loop): a kernel's blocks become resident while its predecessor's last wave runs and
// wait for its completion on the device (pdl_enter) before touching any field.
template <typename R>
__global__ void __launch_bounds__(256) k_roms_zeta(Geo<R> g, RomsArgs<R> a) {
    pdl_enter();
    roms_zeta_at(g, a, tid_flat());
}
template <typename R>
__global__ void __launch_bounds__(256) kb_roms_zeta(const Member<R> *mt, const int2 *bm, RomsArgs<R> a) {
    pdl_enter();
    const MemberAt<R> m = member_at(mt, bm, 256);
    roms_zeta_at(m.g, roms_args_at(a, m.o2), m.p);
}
template <typename R>
__global__ void __launch_bounds__(256) k_roms_mom(Geo<R> g, RomsArgs<R> a) {
    pdl_enter();
    roms_mom_at(g, a, tid_flat());
}
template <typename R>
__global__ void __launch_bounds__(256) kb_roms_mom(const Member<R> *mt, const int2 *bm, RomsArgs<R> a) {
    pdl_enter();
    const MemberAt<R> m = member_at(mt, bm, 256);
    roms_mom_at(m.g, roms_args_at(a, m.o2), m.p);
}
template <typename R>
__global__ void __launch_bounds__(256) k_roms_rhs3d(Geo<R> g, const R *u, const R *v, const R *Hu,
                                                    const R *Hv, const R *Hz, R *ru, R *rv) {
    roms_rhs3d_at(g, u, v, Hu, Hv, Hz, ru, rv, tid_flat());
}
template <typename R>
__global__ void __launch_bounds__(256) kb_roms_rhs3d(const Member<R> *mt, const int2 *bm,
                                                     const R *u, const R *v, const R *Hu,
                                                     const R *Hv, const R *Hz, R *ru, R *rv) {
    const MemberAt<R> m = member_at(mt, bm, 256);
    roms_rhs3d_at(m.g, u + m.o3, v + m.o3, Hu + m.o3, Hv + m.o3, Hz + m.oN, ru + m.o3, rv + m.o3,
                  m.p);
}
template <typename R>
__global__ void __launch_bounds__(256) k_roms_stress3d(Geo<R> g, const R *u, const R *v, R *ru,
                                                       R *rv, const R *sustr, const R *svstr,
                                                       R rdrag2) {
    roms_stress3d_at(g, u, v, ru, rv, sustr, svstr, rdrag2, tid_flat());
}
template <typename R>
__global__ void __launch_bounds__(256) kb_roms_stress3d(const Member<R> *mt, const int2 *bm,
                                                        const R *u, const R *v, R *ru, R *rv,
                                                        const R *sustr, const R *svstr,
                                                        R rdrag2) {
    const MemberAt<R> m = member_at(mt, bm, 256);
    roms_stress3d_at(m.g, u + m.o3, v + m.o3, ru + m.o3, rv + m.o3, sustr + m.o2, svstr + m.o2,
                     rdrag2, m.p);
}
template <typename R>
__global__ void __launch_bounds__(128) k_roms_step3d(Geo<R> g, R *u, R *v, RomsRhs<R> ru,
                                                     RomsRhs<R> rv, R c0, R c1, R c2, R *ubar_n,
                                                     R *vbar_n, R *ubar_s, R *vbar_s, const R *Hz,
                                                     const R *Akv, const R *z_r, const R *W,
                                                     const double *DU, const double *DV, R dt,
                                                     R lamdt) {
    roms_step3d_at(g, u, v, ru, rv, c0, c1, c2, ubar_n, vbar_n, ubar_s, vbar_s, Hz, Akv, z_r, W,
                   DU, DV, dt, lamdt, tid_flat());
}
template <typename R>
__global__ void __launch_bounds__(128) kb_roms_step3d(const Member<R> *mt, const int2 *bm, R *u,
                                                      R *v, RomsRhs<R> ru, RomsRhs<R> rv, R c0,
                                                      R c1, R c2, R *ubar_n, R *vbar_n,
                                                      R *ubar_s, R *vbar_s, const R *Hz,
                                                      const R *Akv, const R *z_r, const R *W,
                                                      const double *DU, const double *DV, R dt,
                                                      R lamdt) {
    const MemberAt<R> m = member_at(mt, bm, 128);
    const long o3 = m.o3, o2 = m.o2;
    const RomsRhs<R> a{ru.r0 + o3, ru.r1 + o3, ru.r2 + o3}, b{rv.r0 + o3, rv.r1 + o3, rv.r2 + o3};
    if (m.p >= m.g.s2) return;
    for (int col = 0; col < 2; ++col)   // the point's U column, then its V column
        roms_step3d_at(m.g, u + o3, v + o3, a, b, c0, c1, c2, ubar_n + o2, vbar_n + o2,
                       ubar_s + o2, vbar_s + o2, Hz + m.oN, Akv + o3, z_r + m.oN, W + o3,
                       DU + o2, DV + o2, dt, lamdt, m.p + col * m.g.s2);
}
template <typename R>
__global__ void __launch_bounds__(256) k_roms_walls3d(Geo<R> g, R *u, R *v) {
    roms_walls3d_at(g, u, v, tid_flat());
}
template <typename R>
__global__ void __launch_bounds__(256) kb_roms_walls3d(const Member<R> *mt, const int2 *bm, R *u,
                                                       R *v) {
    const MemberAt<R> m = member_at(mt, bm, 256);
    roms_walls3d_at(m.g, u + m.o3, v + m.o3, m.p);
}

template <typename R>
cudaError_t Ops<R>::roms_phase(const sf_ctx *c, const RomsArgs<R> &a, cudaStream_t s) {
    if (c->nmem > 1) {
        cudaError_t e = launch_dep(c, kb_roms_zeta<R>, c->nbm_pt, 256, 0, s, mt<R>(c), c->bm_pt, a);
        if (e != cudaSuccess || !a.step) return e;
        return launch_dep(c, kb_roms_mom<R>, c->nbm_pt, 256, 0, s, mt<R>(c), c->bm_pt, a);
    }
    const unsigned nb = blocks_for(c->s2, 256);
    cudaError_t e = launch_dep(c, k_roms_zeta<R>, nb, 256, 0, s, geo(c), a);
    if (e != cudaSuccess || !a.step) return e;
    return launch_dep(c, k_roms_mom<R>, nb, 256, 0, s, geo(c), a);
}
template <typename R>
cudaError_t Ops<R>::roms_stress3d(const sf_ctx *c, const R *u, const R *v, R *ru, R *rv,
                                  const R *sustr, const R *svstr, double rdrag2, cudaStream_t s) {
    if (c->nmem > 1)
        kb_roms_stress3d<R><<<c->nbm_pt, 256, 0, s>>>(mt<R>(c), c->bm_pt, u, v, ru, rv, sustr,
                                                      svstr, (R)rdrag2);
    else
        k_roms_stress3d<R><<<blocks_for(c->s2, 256), 256, 0, s>>>(geo(c), u, v, ru, rv, sustr,
                                                                    svstr, (R)rdrag2);
    return cudaGetLastError();
}
template <typename R>
cudaError_t Ops<R>::roms_rhs3d(const sf_ctx *c, const R *u, const R *v, const R *Huon,
                               const R *Hvom, const R *Hz, R *ru, R *rv, cudaStream_t s) {
    if (c->nmem > 1)
        kb_roms_rhs3d<R><<<c->nbm_pt, 256, 0, s>>>(mt<R>(c), c->bm_pt, u, v, Huon, Hvom, Hz, ru, rv);
    else
        k_roms_rhs3d<R><<<blocks_for(c->s2, 256), 256, 0, s>>>(geo(c), u, v, Huon, Hvom, Hz, ru, rv);
    return cudaGetLastError();
}
template <typename R>
cudaError_t Ops<R>::roms_step3d(const sf_ctx *c, R *u, R *v, const R *const *ru, const R *const *rv,
                                const double *coef, R *ubar_n, R *vbar_n, R *ubar_s, R *vbar_s,
                                const R *Hz, const R *Akv, const R *z_r, const R *W,
                                const double *DU, const double *DV, double dt, double lamdt,
                                cudaStream_t s) {
    const RomsRhs<R> a{ru[0], ru[1], ru[2]}, b{rv[0], rv[1], rv[2]};
    if (c->nmem > 1)
        kb_roms_step3d<R><<<c->nbm_128, 128, 0, s>>>(mt<R>(c), c->bm_128, u, v, a, b, (R)coef[0],
                                                      (R)coef[1], (R)coef[2], ubar_n, vbar_n,
                                                      ubar_s, vbar_s, Hz, Akv, z_r, W, DU, DV,
                                                      (R)dt, (R)lamdt);
    else
        k_roms_step3d<R><<<blocks_for(2 * c->s2, 128), 128, 0, s>>>(geo(c), u, v, a, b, (R)coef[0],
                                                                  (R)coef[1], (R)coef[2], ubar_n,
                                                                  vbar_n, ubar_s, vbar_s, Hz, Akv,
                                                                  z_r, W, DU, DV, (R)dt, (R)lamdt);
    return cudaGetLastError();
}
template <typename R>
cudaError_t Ops<R>::roms_walls3d(const sf_ctx *c, R *u, R *v, cudaStream_t s) {
    if (c->nmem > 1)
        kb_roms_walls3d<R><<<c->nbm_pt, 256, 0, s>>>(mt<R>(c), c->bm_pt, u, v);
    else
        k_roms_walls3d<R><<<blocks_for(c->s2, 256), 256, 0, s>>>(geo(c), u, v);
    return cudaGetLastError();
}

}  // namespace sf
